// Shared device helpers for the fp64 dycore kernels.
//
// Layout: float64 SoA, C order (k, j, i), i fastest.  Mass fields (nz, ny, nx),
// u (nz, ny, nx+1), v (nz, ny+1, nx), w/ph/ww (nz+1, ny, nx), 2-D (ny, nx),
// u-face 2-D (ny, nx+1), v-face 2-D (ny+1, nx).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cmath>

namespace wg {

// Physical constants (src/gpuwrf/dynamics/acoustic_wrf.py:27-75,
// dynamics/core/advance_w.py:28,87-88, runtime/operational_mode.py:202).
constexpr double R_D = 287.0;
constexpr double CP_D = 7.0 * R_D / 2.0;
constexpr double P0 = 100000.0;
constexpr double CPOVCV = CP_D / (CP_D - R_D);
constexpr double CVPM = -(CP_D - R_D) / CP_D;
constexpr double G = 9.81;
constexpr double T0 = 300.0;
constexpr double MIN_ACOUSTIC_ALT = 0.1;
constexpr double W_RERADIUS = 1.0 / 6370.0e3;
constexpr double W_ALPHA = 0.3;
constexpr double W_BETA = 1.0;
constexpr double PD_EPS = 1.0e-20;
constexpr double EMDIV = 0.01;
constexpr double SMDIV = 0.1;
constexpr double MIN_MUTS_FRACTION = 0.5;
constexpr double MIN_MUTS_PA = 1.0;

// Grid geometry and metrics passed by value to every kernel.
struct Grid {
  int nx, ny, nz;
  double rdx, rdy, dx, dy;
  const double *c1h, *c2h, *c3h, *c4h, *c1f, *c2f, *c3f, *c4f;
  const double *dn, *dnw, *rdn, *rdnw, *fnm, *fnp;
  const double *msftx, *msfty, *msfux, *msfuy, *msfvx, *msfvy;
  const double *f, *e, *sina, *cosa;
  // Correctly rounded reciprocals of the map factors (filled once per step),
  // so a division by a map factor is an exact div_rcp.
  const double *rmsftx, *rmsfty, *rmsfux, *rmsfuy, *rmsfvx, *rmsfvy;
  double cf1, cf2, cf3, p_top;
  double cfn, cfn1;  // top-face extrapolation weights (rk_addtend_dry.py:282-288)
};

// The physics merge's w leaves (rk_addtend_dry; NULL = zero) for the w-face kernel.
struct PhysW {
  const double *rw_tendf, *w_save;
  int rk1;
};

// A read-only view of a model state (the reference State leaves the step uses).
struct StateR {
  const double *u, *v, *w, *theta, *p_total, *p_pert, *ph_total, *ph_pert, *mu_total, *mu_pert;
  const double *q[6];
};

struct StateW {
  double *u, *v, *w, *theta, *p_total, *p_pert, *ph_total, *ph_pert, *mu_total, *mu_pert;
  double *q[6];
};

// Element offsets.  Every array of a step has fewer than 2^31 elements (checked
// by wrfgpu_step_params_validate), so the index arithmetic is 32-bit and only
// the final offset is widened.
__device__ __forceinline__ size_t ix3(int k, int j, int i, int ny, int nx) {
  return (size_t)(unsigned)((k * ny + j) * nx + i);
}
__device__ __forceinline__ size_t ix2(int j, int i, int nx) { return (size_t)(unsigned)(j * nx + i); }

// Periodic index wrap; the in-range test keeps the common case branch-only.
__device__ __forceinline__ int wrp(int i, int n) {
  if (i >= 0 && i < n) return i;
  int r = i % n;
  return r < 0 ? r + n : r;
}

__device__ __forceinline__ double sgn(double x) { return (double)((x > 0.0) - (x < 0.0)); }

__device__ __forceinline__ double ld(const double *p, size_t i) { return __ldg(p + i); }
// a float32 intermediate of the mixed-precision variant, widened exactly
__device__ __forceinline__ double ld(const float *p, size_t i) { return (double)__ldg(p + i); }

// jnp.maximum / jnp.minimum semantics are not needed for NaN here; plain compares.
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }

// a / b, correctly rounded, for a divisor b whose reciprocal rb = RN(1/b) is
// known in advance (a literal or a per-launch constant).  This is Markstein's
// correction step (P. Markstein, IBM J. Res. Dev. 34(1):111-119, 1990; J.-M.
// Muller et al., Handbook of Floating-Point Arithmetic, ch. "Division"):
// q0 = RN(a*rb) is within one ulp of a/b, the residual r = a - b*q0 is exact
// in one fma, and RN(q0 + r*rb) is the correctly rounded quotient.  For normal
// operands and quotients the result equals the IEEE quotient a / b bit for bit
// (a zero a may come back as +0 where a / b gives -0); it costs one multiply
// and two fmas instead of a full division sequence.
__device__ __forceinline__ double div_rcp(double a, double b, double rb) {
  const double q0 = __dmul_rn(a, rb);
  const double r = __fma_rn(-b, q0, a);
  return __fma_rn(r, rb, q0);
}
// a / msf[idx] with the map factor's precomputed reciprocal.
__device__ __forceinline__ double div_msf(double a, const double *msf, const double *rmsf, size_t idx) {
  return div_rcp(a, __ldg(msf + idx), __ldg(rmsf + idx));
}
constexpr double R60 = 1.0 / 60.0;
constexpr double R12 = 1.0 / 12.0;
constexpr double RG = 1.0 / G;

// WRF flux5 left-face value (src/gpuwrf/dynamics/flux_advection.py:53-88).
__device__ __forceinline__ double flux5(double qm3, double qm2, double qm1, double q0, double qp1, double qp2,
                                        double vel) {
  double f6 = div_rcp(37.0 * (q0 + qm1) - 8.0 * (qp1 + qm2) + (qp2 + qm3), 60.0, R60);
  double c = div_rcp((qp2 - qm3) - 5.0 * (qp1 - qm2) + 10.0 * (q0 - qm1), 60.0, R60);
  return f6 - sgn(vel) * c;
}

// flux3 with the -sign(vel) upwind correction (flux_advection.py:534-562, 1362-1407).
__device__ __forceinline__ double flux3v(double qkm2, double qkm1, double qk, double qkp1, double vel) {
  double flux4 = div_rcp(7.0 * (qk + qkm1) - (qkp1 + qkm2), 12.0, R12);
  double corr = div_rcp((qkp1 - qkm2) - 3.0 * (qk - qkm1), 12.0, R12);
  return vel * (flux4 + sgn(-vel) * corr);
}

// Advective face fluxes in the arithmetic type F.  F = double: the
// reference's float64 expressions, bit for bit (vel*flux5, flux3v).  F =
// float: the mixed-precision variant -- the stencil is evaluated in FP32 from
// float64 inputs (perturbations are formed in float64 first by the callers)
// and the flux is widened back to float64, so every flux divergence and
// tendency sum stays a float64 accumulation.
template <typename F>
__device__ __forceinline__ double hflux5(double vel, double qm3, double qm2, double qm1, double q0, double qp1,
                                         double qp2) {
  return vel * flux5(qm3, qm2, qm1, q0, qp1, qp2, vel);
}
template <>
__device__ __forceinline__ double hflux5<float>(double vel, double qm3, double qm2, double qm1, double q0, double qp1,
                                                double qp2) {
  const float v = (float)vel, a3 = (float)qm3, a2 = (float)qm2, a1 = (float)qm1, b0 = (float)q0, b1 = (float)qp1,
              b2 = (float)qp2;
  const float f6 = (37.0f * (b0 + a1) - 8.0f * (b1 + a2) + (b2 + a3)) * (1.0f / 60.0f);
  const float c = ((b2 - a3) - 5.0f * (b1 - a2) + 10.0f * (b0 - a1)) * (1.0f / 60.0f);
  const float s = (float)((v > 0.0f) - (v < 0.0f));
  return (double)(v * (f6 - s * c));
}
template <typename F>
__device__ __forceinline__ double vflux3(double vel, double qkm2, double qkm1, double qk, double qkp1) {
  return flux3v(qkm2, qkm1, qk, qkp1, vel);
}
template <>
__device__ __forceinline__ double vflux3<float>(double vel, double qkm2, double qkm1, double qk, double qkp1) {
  const float v = (float)vel, a2 = (float)qkm2, a1 = (float)qkm1, b0 = (float)qk, b1 = (float)qkp1;
  const float flux4 = (7.0f * (b0 + a1) - (b1 + a2)) * (1.0f / 12.0f);
  const float corr = ((b1 - a2) - 3.0f * (b0 - a1)) * (1.0f / 12.0f);
  const float s = (float)((-v > 0.0f) - (-v < 0.0f));
  return (double)(v * (flux4 + s * corr));
}

// flux3 of a horizontal face: flux4 + sign(vel) * correction
// (flux_advection.py:314-317).
template <typename F>
__device__ __forceinline__ double hflux3(double vel, double qm2, double qm1, double q0, double qp1) {
  const double face4 = div_rcp(7.0 * (q0 + qm1) - (qp1 + qm2), 12.0, R12);
  const double corr4 = div_rcp((qp1 - qm2) - 3.0 * (q0 - qm1), 12.0, R12);
  return vel * (face4 + sgn(vel) * corr4);
}
template <>
__device__ __forceinline__ double hflux3<float>(double vel, double qm2, double qm1, double q0, double qp1) {
  const float v = (float)vel, a2 = (float)qm2, a1 = (float)qm1, b0 = (float)q0, b1 = (float)qp1;
  const float face4 = (7.0f * (b0 + a1) - (b1 + a2)) * (1.0f / 12.0f);
  const float corr = ((b1 - a2) - 3.0f * (b0 - a1)) * (1.0f / 12.0f);
  const float s = (float)((v > 0.0f) - (v < 0.0f));
  return (double)(v * (face4 + s * corr));
}

// Flux at face m (between cells m-1 and m) of an axis of n cells under the
// specified-boundary advection degradation (flux_advection.py:288-347):
// flux5 on faces 3..n-3, flux3 on 2 and n-2, 2nd order on 1 and n-1 (with
// the upstream rule for the normal momentum component: the boundary-side
// value is replaced by the interior one under inflow / outflow), zero on
// face 0 (and on face n, the wrap of face 0).  Needs n >= 7, so that every
// tier reads only cells 0..n-1.
template <typename F>
__device__ __forceinline__ double hflux_spec(int m, int n, bool upstream, double vel, double qm3, double qm2,
                                             double qm1, double q0, double qp1, double qp2) {
  if (m >= 3 && m <= n - 3) return hflux5<F>(vel, qm3, qm2, qm1, q0, qp1, qp2);
  if (m == 2 || m == n - 2) return hflux3<F>(vel, qm2, qm1, q0, qp1);
  if (m == 1) return vel * (0.5 * (q0 + ((upstream && q0 < 0.0) ? q0 : qm1)));
  if (m == n - 1) return vel * (0.5 * (qm1 + ((upstream && qm1 > 0.0) ? qm1 : q0)));
  return vel * 0.0;
}

// A specified boundary leaf (time, side W/E/S/N, width, z, side_len)
// (contracts/state.py:96-106) with its time interpolation at one lead
// (boundary_apply.py:329-345: lower / upper time index and weight).
// A boundary leaf (time, side, width, levels, side_len) and its time
// interpolation at one lead (boundary_apply.py:329-345): (lo, hi, alpha)
// resolved on the host, or -- when `lead` is set -- on the device from the
// forecast clock *lead + lead_off, so a step can run with a device-resident
// lead (a traced clock, or one graph replayed with a changing lead).
struct BdyLeaf {
  const double *leaf;
  int ntime, width, side_len, lo, hi;
  double alpha;
  const double *lead;  // device lead in seconds, or nullptr
  double lead_off;     // seconds added to *lead (a stage-end lead)
  double cadence;      // the strips' update cadence in seconds
};

// (lo, hi, alpha) of a leaf at lead L: the reference's clipped floor index of
// L / cadence and its clipped fraction.
__host__ __device__ __forceinline__ void leaf_time_weights(double L, double cadence, int ntime, int &lo, int &hi,
                                                           double &alpha) {
  const int mx = ntime - 1;
  const double li = L / cadence;
  const double fl = floor(li);
  lo = fl < 0.0 ? 0 : (fl > (double)mx ? mx : (int)fl);
  hi = lo + 1 > mx ? mx : lo + 1;
  double a = li - (double)lo;
  alpha = a < 0.0 ? 0.0 : (a > 1.0 ? 1.0 : a);
}

// Strip value of side `side`, width index bb (clamped, boundary_apply.py:528-549),
// level k, tangential index t; nz is the leaf's level count.
__device__ __forceinline__ double strip_at(const BdyLeaf &b, int nz, int side, int bb, int k, int t) {
  bb = bb < 0 ? 0 : (bb > b.width - 1 ? b.width - 1 : bb);
  int lo = b.lo, hi = b.hi;
  double alpha = b.alpha;
  if (b.lead != nullptr) leaf_time_weights(*b.lead + b.lead_off, b.cadence, b.ntime, lo, hi, alpha);
  auto at = [&](int tt) {
    return ld(b.leaf, ((((size_t)tt * 4 + side) * b.width + bb) * nz + k) * b.side_len + t);
  };
  return at(lo) * (1.0 - alpha) + at(hi) * alpha;
}

// Value at (k, j, i) of the leaf written into the outer five rows / columns of
// a (zl, yl, xl) field (boundary_apply.py:948-969: for b = 0..4 the W, E, S, N
// strips in that order, later writes win); 0 off the ring.
__device__ __forceinline__ double ring_target(const BdyLeaf &b, int zl, int yl, int xl, int k, int j, int i) {
  int best = -1, side = 0;
  for (int bb = 0; bb < 5; ++bb) {
    if (i == bb) { best = bb; side = 0; }
    if (i == xl - 1 - bb) { best = bb; side = 1; }
    if (j == bb) { best = bb; side = 2; }
    if (j == yl - 1 - bb) { best = bb; side = 3; }
  }
  if (best < 0) return 0.0;
  return strip_at(b, zl, side, best, k, side < 2 ? j : i);
}

// Dry inverse density from the EOS (acoustic_wrf.py:187-206, qvf = 1).
__device__ __forceinline__ double inv_density(double theta, double p) {
  return (R_D / P0) * theta * 1.0 * pow(dmax(p, 1.0) / P0, CVPM);
}

// EOS pressure inversion (acoustic_wrf.py:209-221, qvf = 1).
__device__ __forceinline__ double pressure_from_theta_alt(double theta, double alt) {
  double argument = (R_D * theta * 1.0) / (P0 * dmax(alt, 1.0e-8));
  return P0 * pow(dmax(argument, 1.0e-12), CPOVCV);
}

// 8-byte asynchronous global->shared copy (cp.async), its group commit and
// the wait for all but the N most recent groups of this thread.
__device__ __forceinline__ void cp_async8(void *smem_dst, const void *gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Hint: pull the row of n doubles starting at p into L2 with one bulk
// prefetch (cp.async.bulk.prefetch.L2).  Only the 16-byte-aligned part that
// lies strictly inside the row is named, so nothing outside it is touched.
__device__ __forceinline__ void l2_prefetch_row(const double *p, int n) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uintptr_t lo = (a + 15) & ~uintptr_t(15);
  const uintptr_t hi = (a + (uintptr_t)n * sizeof(double)) & ~uintptr_t(15);
  if (hi > lo) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((unsigned)(hi - lo)) : "memory");
}

__device__ __forceinline__ double safe12(double x) { return fabs(x) > 1.0e-12 ? x : 1.0e-12; }

}  // namespace wg
