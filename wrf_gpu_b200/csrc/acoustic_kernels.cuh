// Acoustic substep kernels (fp64) and the end-of-stage finish.
//
// One substep is three launches:
//   k_advance_uv               -- advance_uv on every u and v face
//                                 (core/acoustic.py:626-786), face-parallel;
//   k_div_h                    -- the horizontal divergences the columns need;
//   k_column_tiled             -- advance_mu_t (dynamics/mu_t_advance.py),
//                                 advance_w with its Thomas solve
//                                 (core/advance_w.py:293-627) and calc_p_rho
//                                 with smdiv memory (core/calc_p_rho.py:137-183),
//                                 level-parallel per column block (column_tiled.cuh).
// The column kernel writes only its own column and reads neighbours only of
// stage-constant arrays and of u/v (finished by the face kernels), so a
// substep has no intra-kernel race.
#pragma once
#include "dycore_common.cuh"

namespace wg {

// Acoustic work state (operational_mode.py:1996-2166 AcousticCoreState).
struct Acoustic {
  double *u, *v, *w, *ph, *theta_w, *t2ave, *p, *pm1, *al, *ww;  // evolving
  double *mu, *muts, *muave, *mudf;                              // evolving 2-D
  const double *u_tend, *v_tend, *t_tend, *rw_tend, *ph_tend;    // stage tendencies
  const double *alt, *pb, *c2a, *cqu, *cqv, *cqw, *php, *pt1;    // stage constants
  const double *a, *alpha, *gamma, *ww_1;
  const double *mut, *muu, *muv, *muus, *muvs;                   // stage 2-D
  const double *mu_tend;                                         // base mu tendency (nullable)
  const double *u_1, *v_1, *w_save;                              // stage u, v, w (u_save/v_save/w_save)
  const double *theta_s;                                         // stage theta (t_save = theta - 300)
  const double *phb0;                                            // stage base geopotential at face 0 (ny, nx)
};

constexpr int BDY_MAX_ZONE = 16;

struct BdyArgs {
  int active;
  const double *u_target, *v_target;  // work-array targets (u-face / v-face shapes)
  double sub_ratio;                   // strength * dts / dt_full
  int spec_zone, relax_zone;
  // zone_w[d] = min(1, max(0, sub_ratio*0.1*linear(d))) for the relaxation
  // rows d in [spec_zone, relax_zone), filled by set_bdy_weights.
  double zone_w[BDY_MAX_ZONE];
};

inline void set_bdy_weights(BdyArgs &b) {
  auto hmax = [](double x, double y) { return x > y ? x : y; };
  auto hmin = [](double x, double y) { return x < y ? x : y; };
  for (int d = 0; d < BDY_MAX_ZONE; ++d) b.zone_w[d] = 0.0;
  for (int d = b.spec_zone; d < b.relax_zone && d < BDY_MAX_ZONE; ++d) {
    const double linear =
        (b.relax_zone > 1) ? hmax(0.0, (double)(b.spec_zone + b.relax_zone - (d + 1)) / (double)(b.relax_zone - 1)) : 0.0;
    b.zone_w[d] = hmin(1.0, hmax(0.0, b.sub_ratio * 0.1 * linear));
  }
}

// Weight of the per-substep convex blend toward the boundary work target
// (coupling/boundary_apply.py:803-855), DEFAULT_BOUNDARY_CONFIG widths.
__device__ __forceinline__ double relax_weight_u(int j, int i, int y_len, int x_len, const BdyArgs &b) {
  double w = 0.0;
  for (int d = 0; d < b.spec_zone; ++d) {
    if (i == d || i == x_len - 1 - d) w = 1.0;
  }
  for (int d = b.spec_zone; d < b.relax_zone; ++d) {
    if (j >= d + 1 && j < y_len - d - 1 && (i == d || i == x_len - 1 - d)) w = b.zone_w[d];
  }
  return w;
}

__device__ __forceinline__ double relax_weight_v(int j, int i, int y_len, int x_len, const BdyArgs &b) {
  double w = 0.0;
  for (int d = 0; d < b.spec_zone; ++d) {
    if (j == d || j == y_len - 1 - d) w = 1.0;
  }
  for (int d = b.spec_zone; d < b.relax_zone; ++d) {
    if (i >= d && i < x_len - d && (j == d || j == y_len - 1 - d)) w = b.zone_w[d];
  }
  return w;
}

// ---------------------------------------------------------------------------
// advance_uv, one u face (core/acoustic.py:626-735).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void advance_u_face(const Grid &g, const Acoustic &A, double dts, int top_lid,
                                               const BdyArgs &bdy, int i, int j, int k) {
  const int nx = g.nx, ny = g.ny;
  const int nxu = nx + 1;
  const size_t cu = ix3(k, j, i, ny, nxu);
  const size_t f2 = ix2(j, i, nxu);
  double u = A.u[cu] + dts * ld(A.u_tend, cu);
  const int l = (i == 0) ? 0 : i - 1;
  const int r = (i == nx) ? nx - 1 : i;
  auto P = [&](const double *a, int kk, int ic) { return ld(a, ix3(kk, j, ic, ny, nx)); };
  auto PH = [&](int kk, int ic) { return ld(A.ph, ix3(kk, j, ic, ny, nx)); };
  auto PP = [&](int kk, int ic) { return ld(A.p, ix3(kk, j, ic, ny, nx)); };
  auto AL = [&](int kk, int ic) { return ld(A.al, ix3(kk, j, ic, ny, nx)); };
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  const double ph_term = (PH(k + 1, r) - PH(k + 1, l)) + (PH(k, r) - PH(k, l));
  const double p_term = (P(A.alt, k, l) + P(A.alt, k, r)) * (PP(k, r) - PP(k, l));
  const double pb_term = (AL(k, l) + AL(k, r)) * (P(A.pb, k, r) - P(A.pb, k, l));
  const double mass_x = c1 * ld(A.muu, f2) + c2;
  const double msfr = div_msf(ld(g.msfux, f2), g.msfuy, g.rmsfuy, f2);
  double dpx = msfr * 0.5 * g.rdx * mass_x * (ph_term + p_term + pb_term);
  auto ps = [&](int m) { return PP(m, l) + PP(m, r); };
  const double mw_l = ld(A.muts, ix2(j, l, nx)) - ld(A.mut, ix2(j, l, nx));
  const double mw_r = ld(A.muts, ix2(j, r, nx)) - ld(A.mut, ix2(j, r, nx));
  const double bracket = ld(g.rdnw, k) * (dpn_acoustic(g, k + 1, top_lid, ps) - dpn_acoustic(g, k, top_lid, ps)) -
                         0.5 * (c1 * (mw_l + mw_r));
  dpx = dpx + msfr * g.rdx * (P(A.php, k, r) - P(A.php, k, l)) * bracket;
  u = u - dts * ld(A.cqu, cu) * dpx;
  const double md = div_msf(-EMDIV * g.dx * (ld(A.mudf, ix2(j, r, nx)) - ld(A.mudf, ix2(j, l, nx))), g.msfuy, g.rmsfuy, f2);
  u = u + c1 * md;
  if (bdy.active) {
    const double w = relax_weight_u(j, i, ny, nxu, bdy);
    if (w != 0.0) u = u + w * (ld(bdy.u_target, cu) - u);
  }
  A.u[cu] = u;
}

// advance_uv, one v face (core/acoustic.py:737-750).
__device__ __forceinline__ void advance_v_face(const Grid &g, const Acoustic &A, double dts, int top_lid,
                                               const BdyArgs &bdy, int i, int j, int k) {
  const int nx = g.nx, ny = g.ny;
  const int nyv = ny + 1;
  const size_t cv = ix3(k, j, i, nyv, nx);
  const size_t f2 = ix2(j, i, nx);
  double v = A.v[cv] + dts * ld(A.v_tend, cv);
  const int sj = (j == 0) ? 0 : j - 1;
  const int nj = (j == ny) ? ny - 1 : j;
  auto P = [&](const double *a, int kk, int jc) { return ld(a, ix3(kk, jc, i, ny, nx)); };
  auto PH = [&](int kk, int jc) { return ld(A.ph, ix3(kk, jc, i, ny, nx)); };
  auto PP = [&](int kk, int jc) { return ld(A.p, ix3(kk, jc, i, ny, nx)); };
  auto AL = [&](int kk, int jc) { return ld(A.al, ix3(kk, jc, i, ny, nx)); };
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  const double ph_term = (PH(k + 1, nj) - PH(k + 1, sj)) + (PH(k, nj) - PH(k, sj));
  const double p_term = (P(A.alt, k, sj) + P(A.alt, k, nj)) * (PP(k, nj) - PP(k, sj));
  const double pb_term = (AL(k, sj) + AL(k, nj)) * (P(A.pb, k, nj) - P(A.pb, k, sj));
  const double mass_y = c1 * ld(A.muv, f2) + c2;
  const double msfr = div_msf(ld(g.msfvy, f2), g.msfvx, g.rmsfvx, f2);
  double dpy = msfr * 0.5 * g.rdy * mass_y * (ph_term + p_term + pb_term);
  auto ps = [&](int m) { return PP(m, sj) + PP(m, nj); };
  const double mw_s = ld(A.muts, ix2(sj, i, nx)) - ld(A.mut, ix2(sj, i, nx));
  const double mw_n = ld(A.muts, ix2(nj, i, nx)) - ld(A.mut, ix2(nj, i, nx));
  const double bracket = ld(g.rdnw, k) * (dpn_acoustic(g, k + 1, top_lid, ps) - dpn_acoustic(g, k, top_lid, ps)) -
                         0.5 * (c1 * (mw_s + mw_n));
  dpy = dpy + msfr * g.rdy * (P(A.php, k, nj) - P(A.php, k, sj)) * bracket;
  v = v - dts * ld(A.cqv, cv) * dpy;
  const double md = -EMDIV * g.dy * (ld(A.mudf, ix2(nj, i, nx)) - ld(A.mudf, ix2(sj, i, nx))) * ld(g.rmsfvx, f2);
  v = v + c1 * md;
  if (bdy.active) {
    const double w = relax_weight_v(j, i, nyv, nx, bdy);
    if (w != 0.0) v = v + w * (ld(bdy.v_target, cv) - v);
  }
  A.v[cv] = v;
}

// advance_uv on both face kinds of one (k, j, i): the u face at i (j < ny)
// and the v face at j (i < nx).  The two faces read the same mass-point
// neighbourhood (p, al, alt, pb, php, ph, muts, mut, mudf), so one thread
// doing both halves those reads; index space (nx+1) x (ny+1) x nz.
#ifndef WG_UV_KPER
#define WG_UV_KPER 1
#endif
constexpr int UV_KPER = WG_UV_KPER;  // levels per thread (shares the ph / p planes of adjacent levels)

__global__ void k_advance_uv(Grid g, Acoustic A, double dts, int top_lid, BdyArgs bdy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
#pragma unroll
  for (int kk = 0; kk < UV_KPER; ++kk) {
    const int k = blockIdx.z * UV_KPER + kk;
    if (k >= g.nz) break;
    if (i <= g.nx && j < g.ny) advance_u_face(g, A, dts, top_lid, bdy, i, j, k);
    if (i < g.nx && j <= g.ny) advance_v_face(g, A, dts, top_lid, bdy, i, j, k);
  }
}

// ---------------------------------------------------------------------------
// Horizontal parts of advance_mu_t that couple neighbouring columns, one
// thread per cell, after advance_uv: the coupled mass-flux divergence dvdxi
// (dynamics/mu_t_advance.py:186-204) and the horizontal theta flux divergence
// msftx*(0.5*rdy*v_flux + 0.5*rdx*u_flux) (:239-262).  Both are written for
// the interior columns the column kernel updates and read there per level.
// ---------------------------------------------------------------------------
__global__ void k_div_h(Grid g, Acoustic A, int specified, double *dvdxi, double *hdiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nxu = nx + 1, nyv = ny + 1;
  if (i >= nx || j >= ny) return;
  if (specified && !(j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2)) return;
  const size_t c2d = ix2(j, i, nx);
  const double msftx = ld(g.msftx, c2d), msfty = ld(g.msfty, c2d);
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  const double v_n = ld(A.v, ix3(k, j + 1, i, nyv, nx)), v_s = ld(A.v, ix3(k, j, i, nyv, nx));
  const double u_e = ld(A.u, ix3(k, j, i + 1, ny, nxu)), u_w = ld(A.u, ix3(k, j, i, ny, nxu));
  const double vn = v_n + (c1 * ld(A.muv, ix2(j + 1, i, nx)) + c2) * ld(A.v_1, ix3(k, j + 1, i, nyv, nx)) *
                              ld(g.rmsfvx, ix2(j + 1, i, nx));
  const double vs = v_s + (c1 * ld(A.muv, ix2(j, i, nx)) + c2) * ld(A.v_1, ix3(k, j, i, nyv, nx)) *
                              ld(g.rmsfvx, ix2(j, i, nx));
  const double ue = u_e + div_msf((c1 * ld(A.muu, ix2(j, i + 1, nxu)) + c2) * ld(A.u_1, ix3(k, j, i + 1, ny, nxu)),
                                  g.msfuy, g.rmsfuy, ix2(j, i + 1, nxu));
  const double uw = u_w + div_msf((c1 * ld(A.muu, ix2(j, i, nxu)) + c2) * ld(A.u_1, ix3(k, j, i, ny, nxu)),
                                  g.msfuy, g.rmsfuy, ix2(j, i, nxu));
  const size_t c = ix3(k, j, i, ny, nx);
  dvdxi[c] = msftx * msfty * (g.rdy * (vn - vs) + g.rdx * (ue - uw));
  int ie, iw, jn, js;
  if (specified) {
    ie = i + 1; iw = i - 1; jn = j + 1; js = j - 1;
  } else {
    ie = wrp(i + 1, nx); iw = wrp(i - 1, nx); jn = wrp(j + 1, ny); js = wrp(j - 1, ny);
  }
  auto T1 = [&](int jj, int ii2) { return ld(A.theta_s, ix3(k, jj, ii2, ny, nx)) - T0; };
  const double th = T1(j, i);
  const double v_flux = v_n * (T1(jn, i) + th) - v_s * (th + T1(js, i));
  const double u_flux = u_e * (T1(j, ie) + th) - u_w * (th + T1(j, iw));
  hdiv[c] = msftx * (0.5 * g.rdy * v_flux + 0.5 * g.rdx * u_flux);
}

// ---------------------------------------------------------------------------
// Arguments of the column kernel (advance_mu_t + advance_w + calc_p_rho for
// one substep, column_tiled.cuh).
// ---------------------------------------------------------------------------
struct ColArgs {
  double dts, epssm;
  int specified, top_lid, w_damping, damp_opt;
  double dampcoef, zdamp;
  double rzdamp;  // 1/zdamp correctly rounded, 0 when zdamp is 0 or its reciprocal overflows
};

// (x / zdamp) of the Rayleigh ramp, exact either way.
__device__ __forceinline__ double over_zdamp(double x, const ColArgs &c) {
  return c.rzdamp != 0.0 ? div_rcp(x, c.zdamp, c.rzdamp) : x / c.zdamp;
}

}  // namespace wg
