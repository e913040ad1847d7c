// Acoustic substep kernels (fp64) and the end-of-stage finish.
//
// One substep is three launches:
//   k_advance_uv               -- advance_uv on every u and v face
//                                 (core/acoustic.py:626-786), level-marching;
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
  // specified boundary cadence: ring-0 tangential wind work pins from the u / v
  // leaves at the stage-end lead (boundary_apply.py:1251-1296)
  int cad;
  BdyLeaf cad_u, cad_v;
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
// advance_uv (core/acoustic.py:626-786) on both face kinds of one horizontal
// position (i, j), marching up a chunk of UV_KC levels: the u face at i
// (j < ny; acoustic.py:626-735) and the v face at j (i < nx; :737-750).
// Both faces read the mass points C = (jc, ic), W = (jc, i-1) and
// S = (j-1, ic), edge-clamped like the reference's face pairs (u uses W|C,
// v uses S|C).  p and ph of the three points are carried up the chunk in
// registers and the level-invariant 2-D terms are formed once, so a level
// loads only its new plane values; every expression keeps the reference's
// operation order.  Index space (nx+1) x (ny+1) x ceil(nz / UV_KC).
// ---------------------------------------------------------------------------
// levels per thread: timed at 433 x 433 x 50 (bench CUDA events, ms/step):
// 17 (three chunks of 50 levels) 2.80, 13 2.88, 10 2.91, 9 2.95, 25 2.94,
// 50 3.00; 17 with 3 blocks per SM 3.30
#ifndef WG_UV_KC
#define WG_UV_KC 17
#endif
constexpr int UV_KC = WG_UV_KC;
// resident 128-thread blocks per SM requested from the register allocator
// (4: 128 registers; timed at 433 x 433 x 50 against 1 (164 registers) and 5)
#ifndef WG_UV_MINB
#define WG_UV_MINB 4
#endif

// PIN: compile in the boundary cadence's ring-0 tangential wind pins.
template <bool PIN = false>
__global__ void __launch_bounds__(128, WG_UV_MINB) k_advance_uv(Grid g, Acoustic A, double dts, int top_lid, BdyArgs bdy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxu = nx + 1, nyv = ny + 1;
  if (i > nx || j > ny) return;
  const int k0 = blockIdx.z * UV_KC;
  const int k1 = min(k0 + UV_KC, nz);
  const bool du = j < ny, dv = i < nx;
  const int ic = min(i, nx - 1), jc = min(j, ny - 1);
  const int oC = jc * nx + ic, oW = jc * nx + max(i - 1, 0), oS = max(j - 1, 0) * nx + ic;
  const int plane = ny * nx, uplane = ny * nxu, vplane = nyv * nx;
  const int fu = j * nxu + i, fv = j * nx + i;

  // level-invariant parts of the u and v face updates
  double muu = 0.0, msfr_u = 0.0, mwu = 0.0, mdu = 0.0, wu = 0.0;
  if (du) {
    muu = ld(A.muu, fu);
    msfr_u = div_msf(ld(g.msfux, fu), g.msfuy, g.rmsfuy, fu);
    const double mw_l = ld(A.muts, oW) - ld(A.mut, oW);
    const double mw_r = ld(A.muts, oC) - ld(A.mut, oC);
    mwu = mw_l + mw_r;
    mdu = div_msf(-EMDIV * g.dx * (ld(A.mudf, oC) - ld(A.mudf, oW)), g.msfuy, g.rmsfuy, fu);
    if (bdy.active) wu = relax_weight_u(j, i, ny, nxu, bdy);
  }
  double muv = 0.0, msfr_v = 0.0, mwv = 0.0, mdv = 0.0, wv = 0.0;
  if (dv) {
    muv = ld(A.muv, fv);
    msfr_v = div_msf(ld(g.msfvy, fv), g.msfvx, g.rmsfvx, fv);
    const double mw_s = ld(A.muts, oS) - ld(A.mut, oS);
    const double mw_n = ld(A.muts, oC) - ld(A.mut, oC);
    mwv = mw_s + mw_n;
    mdv = -EMDIV * g.dy * (ld(A.mudf, oC) - ld(A.mudf, oS)) * ld(g.rmsfvx, fv);
    if (bdy.active) wv = relax_weight_v(j, i, nyv, nx, bdy);
  }

  // register window: p at k-1 (m) and k (0), ph at k
  const double *pp = A.p, *ph = A.ph;
  int o = k0 * plane;
  double pCm = 0.0, pWm = 0.0, pSm = 0.0;
  if (k0 >= 1) {
    pCm = ld(pp, o - plane + oC); pWm = ld(pp, o - plane + oW); pSm = ld(pp, o - plane + oS);
  }
  double pC0 = ld(pp, o + oC), pW0 = ld(pp, o + oW), pS0 = ld(pp, o + oS);
  double hC0 = ld(ph, o + oC), hW0 = ld(ph, o + oW), hS0 = ld(ph, o + oS);

  // one level's plane values: p and ph one level up, the four mass-point
  // arrays and the two faces' own values
  struct Lvl {
    double pC1, pW1, pS1, hC1, hW1, hS1, altC, altW, altS, alC, alW, alS, pbC, pbW, pbS, phpC, phpW, phpS;
    double u, ut, cqu, v, vt, cqv;
  };
  auto load_lvl = [&](int k, int ok) {
    Lvl L;
    L.pC1 = L.pW1 = L.pS1 = 0.0;
    if (k + 1 < nz) {
      L.pC1 = ld(pp, ok + plane + oC); L.pW1 = ld(pp, ok + plane + oW); L.pS1 = ld(pp, ok + plane + oS);
    }
    L.hC1 = ld(ph, ok + plane + oC); L.hW1 = ld(ph, ok + plane + oW); L.hS1 = ld(ph, ok + plane + oS);
    L.altC = ld(A.alt, ok + oC); L.altW = ld(A.alt, ok + oW); L.altS = ld(A.alt, ok + oS);
    L.alC = ld(A.al, ok + oC); L.alW = ld(A.al, ok + oW); L.alS = ld(A.al, ok + oS);
    L.pbC = ld(A.pb, ok + oC); L.pbW = ld(A.pb, ok + oW); L.pbS = ld(A.pb, ok + oS);
    L.phpC = ld(A.php, ok + oC); L.phpW = ld(A.php, ok + oW); L.phpS = ld(A.php, ok + oS);
    L.u = L.ut = L.cqu = L.v = L.vt = L.cqv = 0.0;
    if (du) {
      const int cu = k * uplane + fu;
      L.u = A.u[cu]; L.ut = ld(A.u_tend, cu); L.cqu = ld(A.cqu, cu);
    }
    if (dv) {
      const int cv = k * vplane + fv;
      L.v = A.v[cv]; L.vt = ld(A.v_tend, cv); L.cqv = ld(A.cqv, cv);
    }
    return L;
  };
  for (int k = k0; k < k1; ++k, o += plane) {
    const Lvl L = load_lvl(k, o);
    const double pC1 = L.pC1, pW1 = L.pW1, pS1 = L.pS1, hC1 = L.hC1, hW1 = L.hW1, hS1 = L.hS1;
    const double altC = L.altC, altW = L.altW, altS = L.altS, alC = L.alC, alW = L.alW, alS = L.alS;
    const double pbC = L.pbC, pbW = L.pbW, pbS = L.pbS, phpC = L.phpC, phpW = L.phpW, phpS = L.phpS;
    const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k), rdnw = ld(g.rdnw, k);
    // extra p levels of the boundary extrapolations: level 2 for the bottom
    // face (k == 0), level nz-3 for a rigid lid's top face (k == nz-1)
    double pCx = 0.0, pWx = 0.0, pSx = 0.0;
    const bool bot = (k == 0), top = (k + 1 == nz) && top_lid;
    if (bot || top) {
      const int ox = (bot ? 2 : nz - 3) * plane;
      pCx = ld(pp, ox + oC); pWx = ld(pp, ox + oW); pSx = ld(pp, ox + oS);
    }
    // dpn_acoustic at faces k+1 (hi) and k (lo) for the pair sums
    // ps(m) = p(m, a) + p(m, C), a = W for u and S for v
    auto dpn_pair = [&](double am, double a0, double a1, double ax, double cm, double c0, double c1v, double cx,
                        double &hi, double &lo) {
      if (k + 1 < nz) hi = 0.5 * (ld(g.fnm, k + 1) * (a1 + c1v) + ld(g.fnp, k + 1) * (a0 + c0));
      else hi = top_lid ? 0.5 * (g.cf1 * (a0 + c0) + g.cf2 * (am + cm) + g.cf3 * (ax + cx)) : 0.0;
      if (bot) lo = 0.5 * (g.cf1 * (a0 + c0) + g.cf2 * (a1 + c1v) + g.cf3 * (ax + cx));
      else lo = 0.5 * (ld(g.fnm, k) * (a0 + c0) + ld(g.fnp, k) * (am + cm));
    };
    if (du) {
      const int cu = k * uplane + fu;
      double u = L.u + dts * L.ut;
      const double ph_term = (hC1 - hW1) + (hC0 - hW0);
      const double p_term = (altW + altC) * (pC0 - pW0);
      const double pb_term = (alW + alC) * (pbC - pbW);
      const double mass_x = c1 * muu + c2;
      double dpx = msfr_u * 0.5 * g.rdx * mass_x * (ph_term + p_term + pb_term);
      double hi, lo;
      dpn_pair(pWm, pW0, pW1, pWx, pCm, pC0, pC1, pCx, hi, lo);
      const double bracket = rdnw * (hi - lo) - 0.5 * (c1 * mwu);
      dpx = dpx + msfr_u * g.rdx * (phpC - phpW) * bracket;
      u = u - dts * L.cqu * dpx;
      u = u + c1 * mdu;
      if (wu != 0.0) u = u + wu * (ld(bdy.u_target, cu) - u);
      if (PIN && bdy.cad && (j == 0 || j == ny - 1)) {
        // tangential u on the S / N rows (core/acoustic.py:777-785)
        const double ms = c1 * ld(A.muus, fu) + c2, mc = c1 * ld(A.muu, fu) + c2;
        u = div_msf(strip_at(bdy.cad_u, nz, j == 0 ? 2 : 3, 0, k, i) * ms - ld(A.u_1, cu) * mc, g.msfuy, g.rmsfuy, fu);
      }
      A.u[cu] = u;
    }
    if (dv) {
      const int cv = k * vplane + fv;
      double v = L.v + dts * L.vt;
      const double ph_term = (hC1 - hS1) + (hC0 - hS0);
      const double p_term = (altS + altC) * (pC0 - pS0);
      const double pb_term = (alS + alC) * (pbC - pbS);
      const double mass_y = c1 * muv + c2;
      double dpy = msfr_v * 0.5 * g.rdy * mass_y * (ph_term + p_term + pb_term);
      double hi, lo;
      dpn_pair(pSm, pS0, pS1, pSx, pCm, pC0, pC1, pCx, hi, lo);
      const double bracket = rdnw * (hi - lo) - 0.5 * (c1 * mwv);
      dpy = dpy + msfr_v * g.rdy * (phpC - phpS) * bracket;
      v = v - dts * L.cqv * dpy;
      v = v + c1 * mdv;
      if (wv != 0.0) v = v + wv * (ld(bdy.v_target, cv) - v);
      if (PIN && bdy.cad && (i == 0 || i == nx - 1) && j >= 1 && j <= ny - 1) {
        // tangential v on the W / E columns
        const double ms = c1 * ld(A.muvs, fv) + c2, mc = c1 * ld(A.muv, fv) + c2;
        v = div_msf(strip_at(bdy.cad_v, nz, i == 0 ? 0 : 1, 0, k, j) * ms - ld(A.v_1, cv) * mc, g.msfvx, g.rmsfvx, fv);
      }
      A.v[cv] = v;
    }
    pCm = pC0; pWm = pW0; pSm = pS0;
    pC0 = pC1; pW0 = pW1; pS0 = pS1;
    hC0 = hC1; hW0 = hW1; hS0 = hS1;
  }
}

// ---------------------------------------------------------------------------
// Horizontal parts of advance_mu_t that couple neighbouring columns, one
// thread per cell, after advance_uv: the coupled mass-flux divergence dvdxi
// (dynamics/mu_t_advance.py:186-204) and the horizontal theta flux divergence
// msftx*(0.5*rdy*v_flux + 0.5*rdx*u_flux) (:239-262).  Both are written for
// the interior columns the column kernel updates and read there per level.
// ---------------------------------------------------------------------------
// 16 resident blocks of 128 per SM (32 registers, full occupancy): timed at
// 433 x 433 x 50, 1.316 vs 1.388 ms/step with the compiler's 40 registers.
#ifndef WG_DIVH_MINB
#define WG_DIVH_MINB 16
#endif
#if WG_DIVH_MINB > 0
#define WG_DIVH_BOUNDS __launch_bounds__(128, WG_DIVH_MINB)
#else
#define WG_DIVH_BOUNDS
#endif
__global__ void WG_DIVH_BOUNDS k_div_h(Grid g, Acoustic A, int specified, double *dvdxi, double *hdiv) {
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
  // specified boundary cadence: ring-0 pins of mu / muts / muave and the work
  // theta from the leaves at the stage-end lead (operational_mode.py:1984-2029;
  // core/acoustic.py:902-915)
  int cad;
  BdyLeaf cad_mu, cad_th;
  // ring-0 work ph pin after advance_w (spec_bdyupdate_ph, core/acoustic.py:1059-1071):
  // the cadence's at the stage-end lead, the nested child's at the step's lead
  // (operational_mode.py:1961-1968)
  int ph_pin;
  BdyLeaf cad_ph;
  const double *ph_save;  // stage ph' (the work ph's reference)
  const double *mub;      // base dry mass
};

// (x / zdamp) of the Rayleigh ramp, exact either way.
__device__ __forceinline__ double over_zdamp(double x, const ColArgs &c) {
  return c.rzdamp != 0.0 ? div_rcp(x, c.zdamp, c.rzdamp) : x / c.zdamp;
}

}  // namespace wg
