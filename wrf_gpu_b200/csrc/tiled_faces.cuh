// Tiled u/v/w-face stage kernels and the level-parallel transport kernel.
//
// The flux-form momentum advection (flux_advection.py:1131-1329) reads its
// horizontal stencils from shared-memory plane tiles (periodic wrap applied
// once per staged element); the large-step PGF, Coriolis, pg_buoy_w and
// rhs_ph terms read global memory (L1-cached neighbours).  The wrap face
// (i = nx for u, j = ny for v) takes the global-load advection path, which is
// the reference's periodic copy of face 0.  Arithmetic order is unchanged.
#pragma once
#include "dycore_common.cuh"
#include "stage_kernels.cuh"
#include "tiled_stencils.cuh"

namespace wg {

// Resident blocks per SM requested for the face kernels (register budget).
// (per kernel; chosen by timing each at 433 x 433 x 50: fewer registers and
// more resident warps hide more of the tile loads' latency, up to the point
// where spills cost more than the warps gain)
#ifndef WG_UFACE_MINB
#define WG_UFACE_MINB 5
#endif
#ifndef WG_VFACE_MINB
#define WG_VFACE_MINB 6
#endif
#ifndef WG_WFACE_MINB
#define WG_WFACE_MINB 5
#endif

// Staged inputs of the u faces' large-step PGF (rk_addtend_dry.py:232-362):
// for the block's rows and the mass points i0-1 .. i0+TSX-1 (clamped into
// the domain, the faces' l = max(i-1, 0) and r = min(i, nx-1)), alt, al, pb,
// php and qtot at level k, ph' at levels k and k+1, p' at the three levels
// lev0 .. lev0+2 that dpn at faces k and k+1 reads, and mu', mu.
constexpr int PGF_W = TSX + 1;
enum { PGF_ALT, PGF_AL, PGF_PB, PGF_PHP, PGF_QT, PGF_PH0, PGF_PH1, PGF_P0, PGF_P1, PGF_P2, PGF_MUP, PGF_MUT,
       PGF_U_N };

__device__ __forceinline__ void load_pgf_u(const Grid &g, const StateR &s, const Diag &d, int k, int lev0, int i0,
                                           int j0, double (*spg)[TSY][PGF_W]) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  for (int e = threadIdx.y * TSX + threadIdx.x; e < TSY * PGF_W; e += TSX * TSY) {
    const int r = e / PGF_W, cc = e - r * PGF_W;
    const int jj = j0 + r;
    if (jj >= ny) continue;
    int ic = i0 - 1 + cc;
    ic = ic < 0 ? 0 : (ic > nx - 1 ? nx - 1 : ic);
    auto L3 = [&](const double *a, int kk) { return ld(a, ix3(kk, jj, ic, ny, nx)); };
    spg[PGF_ALT][r][cc] = L3(d.alt_raw, k);
    spg[PGF_AL][r][cc] = L3(d.al_ls, k);
    spg[PGF_PB][r][cc] = L3(d.pb, k);
    spg[PGF_PHP][r][cc] = L3(d.php_ls, k);
    spg[PGF_QT][r][cc] = L3(d.qtot, k);
    spg[PGF_PH0][r][cc] = L3(s.ph_pert, k);
    spg[PGF_PH1][r][cc] = L3(s.ph_pert, k + 1);
    for (int q = 0; q < 3; ++q)
      if (lev0 + q < nz) spg[PGF_P0 + q][r][cc] = L3(s.p_pert, lev0 + q);
    spg[PGF_MUP][r][cc] = ld(s.mu_pert, ix2(jj, ic, nx));
    spg[PGF_MUT][r][cc] = ld(s.mu_total, ix2(jj, ic, nx));
  }
}

// Advection of u at collapsed face ii from global loads (the periodic wrap face).
template <typename F>
__device__ __forceinline__ double u_adv_global(const Grid &g, const StateR &s, const double *ru, const double *rv,
                                               const double *rom, int k, int j, int ii) {
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxu = nx + 1;
  auto uf = [&](int kk, int jj, int mm) { return ld(s.u, ix3(kk, wrp(jj, ny), wrp(mm, nx), ny, nxu)); };
  auto fqx = [&](int m) {
    int rm = wrp(m, nx);
    double vel = 0.5 * (ld(ru, ix3(k, j, rm, ny, nx)) + ld(ru, ix3(k, j, wrp(rm - 1, nx), ny, nx)));
    return hflux5<F>(vel, uf(k, j, rm - 3), uf(k, j, rm - 2), uf(k, j, rm - 1), uf(k, j, rm), uf(k, j, rm + 1),
                       uf(k, j, rm + 2));
  };
  const double msfux_c = ld(g.msfux, ix2(j, ii, nxu));
  double tend = -msfux_c * g.rdx * (fqx(ii + 1) - fqx(ii));
  if (ny > 1) {
    auto fqy = [&](int n) {
      int rn = wrp(n, ny);
      double vel = 0.5 * (ld(rv, ix3(k, rn, ii, ny, nx)) + ld(rv, ix3(k, rn, wrp(ii - 1, nx), ny, nx)));
      return hflux5<F>(vel, uf(k, rn - 3, ii), uf(k, rn - 2, ii), uf(k, rn - 1, ii), uf(k, rn, ii), uf(k, rn + 1, ii),
                         uf(k, rn + 2, ii));
    };
    tend = tend - msfux_c * g.rdy * (fqy(j + 1) - fqy(j));
  }
  auto romq = [&](int m) { return 0.5 * (ld(rom, ix3(m, j, ii, ny, nx)) + ld(rom, ix3(m, j, wrp(ii - 1, nx), ny, nx))); };
  auto q = [&](int kk) { return ld(s.u, ix3(kk, j, ii, ny, nxu)); };
  const double v1 = (k + 1 <= nz - 1) ? vflux3_at<F>(g, k + 1, romq(k + 1), q) : 0.0;
  const double v0 = (k >= 1) ? vflux3_at<F>(g, k, romq(k), q) : 0.0;
  return tend + (-ld(g.rdnw, k)) * (v1 - v0);
}

// Advection of v at collapsed face jj from global loads (the periodic wrap face).
template <typename F>
__device__ __forceinline__ double v_adv_global(const Grid &g, const StateR &s, const double *ru, const double *rv,
                                               const double *rom, int k, int jj, int i) {
  const int nx = g.nx, ny = g.ny, nz = g.nz, nyv = ny + 1;
  auto vf = [&](int kk, int jv, int ic) { return ld(s.v, ix3(kk, wrp(jv, ny), wrp(ic, nx), nyv, nx)); };
  const double msfvy_c = ld(g.msfvy, ix2(jj, i, nx));
  const double msfvx_c = ld(g.msfvx, ix2(jj, i, nx));
  auto fqx = [&](int m) {
    int rm = wrp(m, nx);
    double vel = 0.5 * (ld(ru, ix3(k, jj, rm, ny, nx)) + ld(ru, ix3(k, wrp(jj - 1, ny), rm, ny, nx)));
    return hflux5<F>(vel, vf(k, jj, rm - 3), vf(k, jj, rm - 2), vf(k, jj, rm - 1), vf(k, jj, rm), vf(k, jj, rm + 1),
                       vf(k, jj, rm + 2));
  };
  double tend = -msfvy_c * g.rdx * (fqx(i + 1) - fqx(i));
  auto fqy = [&](int n) {
    int rn = wrp(n, ny);
    double vel = 0.5 * (ld(rv, ix3(k, rn, i, ny, nx)) + ld(rv, ix3(k, wrp(rn - 1, ny), i, ny, nx)));
    return hflux5<F>(vel, vf(k, rn - 3, i), vf(k, rn - 2, i), vf(k, rn - 1, i), vf(k, rn, i), vf(k, rn + 1, i),
                       vf(k, rn + 2, i));
  };
  tend = tend - msfvy_c * g.rdy * (fqy(jj + 1) - fqy(jj));
  auto romq = [&](int m) { return 0.5 * (ld(rom, ix3(m, jj, i, ny, nx)) + ld(rom, ix3(m, wrp(jj - 1, ny), i, ny, nx))); };
  auto q = [&](int kk) { return ld(s.v, ix3(kk, jj, i, nyv, nx)); };
  const double v1 = (k + 1 <= nz - 1) ? vflux3_at<F>(g, k + 1, romq(k + 1), q) : 0.0;
  const double v0 = (k >= 1) ? vflux3_at<F>(g, k, romq(k), q) : 0.0;
  return tend + div_rcp(msfvy_c, msfvx_c, ld(g.rmsfvx, ix2(jj, i, nx))) * ((-ld(g.rdnw, k)) * (v1 - v0));
}

// ---------------------------------------------------------------------------
// u faces, tiled advection.  Grid over faces 0..nx.
// ---------------------------------------------------------------------------
template <typename F, bool DEG>
__global__ void __launch_bounds__(TSX *TSY, WG_UFACE_MINB) k_uface_tiled(Grid g, StateR s, StateR ref, const double *ru,
                                                           const double *rv, const double *rom, Diag d,
                                                           const double *muu, const double *muus,
                                                           const double *base_u, int top_lid, int run_boundary,
                                                           UFaceOut o) {
  constexpr bool deg = DEG;  // the specified-boundary advection degradation
  using TQ = Tile<3, 3>;
  using TR = Tile<1, 0>;
  using TV = Tile<1, 1>;
  __shared__ double su[TQ::N];
  __shared__ double sru[TR::N];
  __shared__ double srv[TV::N];
  // the large-step PGF's mass-point inputs of the block's faces (PGF_U_*),
  // staged with the advection tiles so their loads are in flight together
  __shared__ double spg[PGF_U_N][TSY][PGF_W];
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxu = nx + 1;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * TSX, j0 = blockIdx.y * TSY, k = blockIdx.z;
  const int i = i0 + tx, j = j0 + ty;
  // levels of the p' staged for dpn at faces k and k+1
  const int lev0 = k == 0 ? 0 : k - 1;
  // (the specified degradation reads the real east face u(nx): no x wrap)
  load_tile<3, 3>(su, s.u + (size_t)k * ny * nxu, nxu, i0, j0, deg ? nx + 1 : nx, ny, 0.0);
  load_tile<1, 0>(sru, ru + (size_t)k * ny * nx, nx, i0, j0, nx, ny, 0.0);
  load_tile<1, 1>(srv, rv + (size_t)k * ny * nx, nx, i0, j0, nx, ny, 0.0);
  load_pgf_u(g, s, d, k, lev0, i0, j0, spg);
  __syncthreads();
  if (i > nx || j >= ny) return;
  const size_t cu = ix3(k, j, i, ny, nxu);
  double tend;
  if (deg && (i == 0 || i == nx)) {
    tend = 0.0;  // the specified degradation updates u faces 1..nx-1 only (flux_advection.py:1177-1182)
  } else if (i < nx) {
    auto Q = [&](int r, int cc) { return su[(r + 3) * TQ::W + (cc + 3)]; };
    auto RU = [&](int cc) { return sru[ty * TR::W + (cc + 1)]; };
    auto RV = [&](int r, int cc) { return srv[(r + 1) * TV::W + (cc + 1)]; };
    // full-face coupled u at the domain-edge faces 0 and nx
    // (couple_uv_specified, flux_advection.py:364-391: edge-padded face mass)
    auto ru_edge = [&](int ie) {
      const double mu_e = (ie == 0) ? 0.5 * (ld(s.mu_total, ix2(j, 0, nx)) + ld(s.mu_total, ix2(j, 0, nx)))
                                    : ld(s.mu_total, ix2(j, nx - 1, nx));
      return div_msf((ld(g.c1h, k) * mu_e + ld(g.c2h, k)) * ld(s.u, ix3(k, j, ie, ny, nxu)), g.msfuy, g.rmsfuy,
                     ix2(j, ie, nxu));
    };
    auto fqx = [&](int m) {
      double vel = 0.5 * (RU(m) + RU(m - 1));
      if (deg) {
        const int gm = i0 + m;
        if (gm == 1) vel = 0.5 * (RU(m) + ru_edge(0));
        else if (gm == nx) vel = 0.5 * (ru_edge(nx) + RU(m - 1));
        return hflux_spec<F>(gm, nx + 1, true, vel, Q(ty, m - 3), Q(ty, m - 2), Q(ty, m - 1), Q(ty, m), Q(ty, m + 1),
                             Q(ty, m + 2));
      }
      return hflux5<F>(vel, Q(ty, m - 3), Q(ty, m - 2), Q(ty, m - 1), Q(ty, m), Q(ty, m + 1), Q(ty, m + 2));
    };
    const double msfux_c = ld(g.msfux, ix2(j, i, nxu));
    tend = -msfux_c * g.rdx * (fqx(tx + 1) - fqx(tx));
    if (ny > 1) {
      auto fqy = [&](int r) {
        const double vel = 0.5 * (RV(r, tx) + RV(r, tx - 1));
        if (deg)
          return hflux_spec<F>(j0 + r, ny, false, vel, Q(r - 3, tx), Q(r - 2, tx), Q(r - 1, tx), Q(r, tx),
                               Q(r + 1, tx), Q(r + 2, tx));
        return hflux5<F>(vel, Q(r - 3, tx), Q(r - 2, tx), Q(r - 1, tx), Q(r, tx), Q(r + 1, tx), Q(r + 2, tx));
      };
      const bool yin = !deg || (j >= 1 && j <= ny - 2);
      tend = tend - msfux_c * g.rdy * (yin ? (fqy(ty + 1) - fqy(ty)) : 0.0);
    }
    const int im = wrp(i - 1, nx);
    auto romq = [&](int m) { return 0.5 * (ld(rom, ix3(m, j, i, ny, nx)) + ld(rom, ix3(m, j, im, ny, nx))); };
    auto q = [&](int kk) { return ld(s.u, ix3(kk, j, i, ny, nxu)); };
    const double v1 = (k + 1 <= nz - 1) ? vflux3_at<F>(g, k + 1, romq(k + 1), q) : 0.0;
    const double v0 = (k >= 1) ? vflux3_at<F>(g, k, romq(k), q) : 0.0;
    tend = tend + (-ld(g.rdnw, k)) * (v1 - v0);
  } else {
    tend = u_adv_global<F>(g, s, ru, rv, rom, k, j, 0);
  }
  const int l = (i == 0) ? 0 : i - 1;
  const int r = (i == nx) ? nx - 1 : i;
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  double u_t;
  if (base_u != nullptr) {
    const double mu_l = ld(s.mu_total, ix2(j, l, nx)), mu_r = ld(s.mu_total, ix2(j, r, nx));
    const double muu_a = (i == 0) ? mu_l : (i == nx ? mu_r : 0.5 * (mu_l + mu_r));
    u_t = ld(base_u, cu) * (c1 * muu_a + c2) + tend;
  } else {
    u_t = tend;
  }
  {
    // staged values at the mass point ic (l or r) of this thread's row
    auto S = [&](int slot, int ic) { return spg[slot][ty][ic - i0 + 1]; };
    const double ph_term = (S(PGF_PH1, r) - S(PGF_PH1, l)) + (S(PGF_PH0, r) - S(PGF_PH0, l));
    const int pk = PGF_P0 + (k - lev0);
    const double p_term = (S(PGF_ALT, l) + S(PGF_ALT, r)) * (S(pk, r) - S(pk, l));
    const double pb_term = (S(PGF_AL, l) + S(PGF_AL, r)) * (S(PGF_PB, r) - S(PGF_PB, l));
    const double mp_l = S(PGF_MUP, l), mp_r = S(PGF_MUP, r);
    const double mt_l = (S(PGF_MUT, l) - mp_l) + mp_l;
    const double mt_r = (S(PGF_MUT, r) - mp_r) + mp_r;
    const double mass_u = c1 * (0.5 * (mt_l + mt_r)) + c2;
    const double msf_u = div_msf(ld(g.msfux, ix2(j, i, nxu)), g.msfuy, g.rmsfuy, ix2(j, i, nxu));
    double dpx = msf_u * 0.5 * g.rdx * mass_u * (ph_term + p_term + pb_term);
    auto ps = [&](int m) { return S(PGF_P0 + (m - lev0), l) + S(PGF_P0 + (m - lev0), r); };
    const double bracket = ld(g.rdnw, k) * (dpn_large(g, k + 1, top_lid, ps) - dpn_large(g, k, top_lid, ps)) -
                           0.5 * (c1 * (mp_l + mp_r));
    dpx = dpx + msf_u * g.rdx * (S(PGF_PHP, r) - S(PGF_PHP, l)) * bracket;
    const double cqu = 1.0 / (1.0 + 0.5 * (S(PGF_QT, l) + S(PGF_QT, r)));
    u_t = u_t + (-cqu) * dpx;
    o.cqu[cu] = cqu;
  }
  {
    auto mu2 = [&](int jj, int ic) { return ld(s.mu_total, ix2(jj, ic, nx)); };
    auto rvq = [&](int jv, int ic) {
      const int js = (jv == 0) ? 0 : jv - 1, jn = (jv == ny) ? ny - 1 : jv;
      const double muv_c = 0.5 * (mu2(js, ic) + mu2(jn, ic));
      return div_msf(ld(s.v, ix3(k, jv, ic, ny + 1, nx)) * (c1 * muv_c + c2), g.msfvx, g.rmsfvx, ix2(jv, ic, nx));
    };
    auto rwq = [&](int kf, int ic) {
      return ld(s.w, ix3(kf, j, ic, ny, nx)) * (ld(g.c1f, kf) * mu2(j, ic) + ld(g.c2f, kf)) /
             ld(g.msfty, ix2(j, ic, nx));
    };
    const double f_u = 0.5 * (ld(g.f, ix2(j, l, nx)) + ld(g.f, ix2(j, r, nx)));
    const double e_u = 0.5 * (ld(g.e, ix2(j, l, nx)) + ld(g.e, ix2(j, r, nx)));
    const double cosa_u = 0.5 * (ld(g.cosa, ix2(j, l, nx)) + ld(g.cosa, ix2(j, r, nx)));
    const double msf_u = div_msf(ld(g.msfux, ix2(j, i, nxu)), g.msfuy, g.rmsfuy, ix2(j, i, nxu));
    double ru_cor = 0.0;
    if (f_u != 0.0 || e_u != 0.0) {
      const double rv_quad = 0.25 * (rvq(j, l) + rvq(j, r) + rvq(j + 1, l) + rvq(j + 1, r));
      ru_cor = msf_u * f_u * rv_quad;
      const double rw_quad = 0.25 * (rwq(k, l) + rwq(k + 1, l) + rwq(k, r) + rwq(k + 1, r));
      ru_cor = ru_cor - e_u * cosa_u * rw_quad;
    } else {
      // f = e = 0 (e.g. idealized frames): the products are exact zeros; keep
      // the reference's (+/-)0 arithmetic by multiplying the zero factors.
      ru_cor = msf_u * f_u * 0.0;
      ru_cor = ru_cor - e_u * cosa_u * 0.0;
    }
    if (run_boundary && (i == 0 || i == nx)) ru_cor = ru_cor * 0.0;
    u_t = u_t + ru_cor;
  }
  o.u_tend[cu] = u_t;
  const size_t f2 = ix2(j, i, nxu);
  const double mass_ref = c1 * ld(muus, f2) + c2;
  const double mass_cur = c1 * ld(muu, f2) + c2;
  o.u_w[cu] = div_msf(mass_ref * ld(ref.u, cu) - mass_cur * ld(s.u, cu), g.msfuy, g.rmsfuy, f2);
}

// ---------------------------------------------------------------------------
// v faces, tiled advection.  Grid over faces 0..ny.
// ---------------------------------------------------------------------------
template <typename F, bool DEG>
__global__ void __launch_bounds__(TSX *TSY, WG_VFACE_MINB) k_vface_tiled(Grid g, StateR s, StateR ref, const double *ru,
                                                           const double *rv, const double *rom, Diag d,
                                                           const double *muv, const double *muvs,
                                                           const double *base_v, int top_lid, int run_boundary,
                                                           VFaceOut o) {
  constexpr bool deg = DEG;  // the specified-boundary advection degradation
  using TQ = Tile<3, 3>;
  using TR = Tile<1, 1>;
  using TV = Tile<0, 1>;
  __shared__ double sv[TQ::N];
  __shared__ double sru[TR::N];
  __shared__ double srv[TV::N];
  const int nx = g.nx, ny = g.ny, nz = g.nz, nyv = ny + 1;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * TSX, j0 = blockIdx.y * TSY, k = blockIdx.z;
  const int i = i0 + tx, j = j0 + ty;
  // (the specified degradation reads the real north face v(ny): no y wrap)
  load_tile<3, 3>(sv, s.v + (size_t)k * nyv * nx, nx, i0, j0, nx, deg ? ny + 1 : ny, 0.0);
  load_tile<1, 1>(sru, ru + (size_t)k * ny * nx, nx, i0, j0, nx, ny, 0.0);
  load_tile<0, 1>(srv, rv + (size_t)k * ny * nx, nx, i0, j0, nx, ny, 0.0);
  __syncthreads();
  if (i >= nx || j > ny) return;
  const size_t cv = ix3(k, j, i, nyv, nx);
  double tend;
  if (deg && (j == 0 || j == ny)) {
    tend = 0.0;  // the specified degradation updates v rows 1..ny-1 only (flux_advection.py:1250-1254)
  } else if (j < ny) {
    auto Q = [&](int r, int cc) { return sv[(r + 3) * TQ::W + (cc + 3)]; };
    auto RU = [&](int r, int cc) { return sru[(r + 1) * TR::W + (cc + 1)]; };
    auto RV = [&](int r) { return srv[(r + 1) * TV::W + tx]; };
    const double msfvy_c = ld(g.msfvy, ix2(j, i, nx));
    const double msfvx_c = ld(g.msfvx, ix2(j, i, nx));
    auto fqx = [&](int m) {
      const double vel = 0.5 * (RU(ty, m) + RU(ty - 1, m));
      if (deg)
        return hflux_spec<F>(i0 + m, nx, false, vel, Q(ty, m - 3), Q(ty, m - 2), Q(ty, m - 1), Q(ty, m),
                             Q(ty, m + 1), Q(ty, m + 2));
      return hflux5<F>(vel, Q(ty, m - 3), Q(ty, m - 2), Q(ty, m - 1), Q(ty, m), Q(ty, m + 1), Q(ty, m + 2));
    };
    const bool xin = !deg || (i >= 1 && i <= nx - 2);
    tend = -msfvy_c * g.rdx * (xin ? (fqx(tx + 1) - fqx(tx)) : 0.0);
    // full-face coupled v at the domain-edge rows 0 and ny (flux_advection.py:364-391)
    auto rv_edge = [&](int je) {
      const double mu_e = (je == 0) ? 0.5 * (ld(s.mu_total, ix2(0, i, nx)) + ld(s.mu_total, ix2(0, i, nx)))
                                    : ld(s.mu_total, ix2(ny - 1, i, nx));
      return div_msf((ld(g.c1h, k) * mu_e + ld(g.c2h, k)) * ld(s.v, ix3(k, je, i, nyv, nx)), g.msfvx, g.rmsfvx,
                     ix2(je, i, nx));
    };
    auto fqy = [&](int r) {
      double vel = 0.5 * (RV(r) + RV(r - 1));
      if (deg) {
        const int gr = j0 + r;
        if (gr == 1) vel = 0.5 * (RV(r) + rv_edge(0));
        else if (gr == ny) vel = 0.5 * (rv_edge(ny) + RV(r - 1));
        return hflux_spec<F>(gr, ny + 1, true, vel, Q(r - 3, tx), Q(r - 2, tx), Q(r - 1, tx), Q(r, tx), Q(r + 1, tx),
                             Q(r + 2, tx));
      }
      return hflux5<F>(vel, Q(r - 3, tx), Q(r - 2, tx), Q(r - 1, tx), Q(r, tx), Q(r + 1, tx), Q(r + 2, tx));
    };
    tend = tend - msfvy_c * g.rdy * (fqy(ty + 1) - fqy(ty));
    const int jm = wrp(j - 1, ny);
    auto romq = [&](int m) { return 0.5 * (ld(rom, ix3(m, j, i, ny, nx)) + ld(rom, ix3(m, jm, i, ny, nx))); };
    auto q = [&](int kk) { return ld(s.v, ix3(kk, j, i, nyv, nx)); };
    const double v1 = (k + 1 <= nz - 1) ? vflux3_at<F>(g, k + 1, romq(k + 1), q) : 0.0;
    const double v0 = (k >= 1) ? vflux3_at<F>(g, k, romq(k), q) : 0.0;
    tend = tend + div_rcp(msfvy_c, msfvx_c, ld(g.rmsfvx, ix2(j, i, nx))) * ((-ld(g.rdnw, k)) * (v1 - v0));
  } else {
    tend = v_adv_global<F>(g, s, ru, rv, rom, k, 0, i);
  }
  const int sj = (j == 0) ? 0 : j - 1;
  const int nj = (j == ny) ? ny - 1 : j;
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  double v_t;
  if (base_v != nullptr) {
    const double mu_s = ld(s.mu_total, ix2(sj, i, nx)), mu_n = ld(s.mu_total, ix2(nj, i, nx));
    const double muv_a = (j == 0) ? mu_s : (j == ny ? mu_n : 0.5 * (mu_s + mu_n));
    v_t = ld(base_v, cv) * (c1 * muv_a + c2) + tend;
  } else {
    v_t = tend;
  }
  {
    auto P = [&](const double *a, int kk, int jc) { return ld(a, ix3(kk, jc, i, ny, nx)); };
    const double ph_term = (P(s.ph_pert, k + 1, nj) - P(s.ph_pert, k + 1, sj)) + (P(s.ph_pert, k, nj) - P(s.ph_pert, k, sj));
    const double p_term = (P(d.alt_raw, k, sj) + P(d.alt_raw, k, nj)) * (P(s.p_pert, k, nj) - P(s.p_pert, k, sj));
    const double pb_term = (P(d.al_ls, k, sj) + P(d.al_ls, k, nj)) * (P(d.pb, k, nj) - P(d.pb, k, sj));
    const double mp_s = ld(s.mu_pert, ix2(sj, i, nx)), mp_n = ld(s.mu_pert, ix2(nj, i, nx));
    const double mt_s = (ld(s.mu_total, ix2(sj, i, nx)) - mp_s) + mp_s;
    const double mt_n = (ld(s.mu_total, ix2(nj, i, nx)) - mp_n) + mp_n;
    const double mass_v = c1 * (0.5 * (mt_s + mt_n)) + c2;
    const double msf_v = div_msf(ld(g.msfvy, ix2(j, i, nx)), g.msfvx, g.rmsfvx, ix2(j, i, nx));
    double dpy = msf_v * 0.5 * g.rdy * mass_v * (ph_term + p_term + pb_term);
    auto ps = [&](int m) { return P(s.p_pert, m, sj) + P(s.p_pert, m, nj); };
    const double bracket = ld(g.rdnw, k) * (dpn_large(g, k + 1, top_lid, ps) - dpn_large(g, k, top_lid, ps)) -
                           0.5 * (c1 * (mp_s + mp_n));
    dpy = dpy + msf_v * g.rdy * (P(d.php_ls, k, nj) - P(d.php_ls, k, sj)) * bracket;
    const double cqv = 1.0 / (1.0 + 0.5 * (P(d.qtot, k, sj) + P(d.qtot, k, nj)));
    v_t = v_t + (-cqv) * dpy;
    o.cqv[cv] = cqv;
  }
  {
    auto mu2 = [&](int jc, int ic) { return ld(s.mu_total, ix2(jc, ic, nx)); };
    auto ruq = [&](int jc, int iu) {
      const int il = (iu == 0) ? 0 : iu - 1, ir = (iu == nx) ? nx - 1 : iu;
      const double muu_c = 0.5 * (mu2(jc, il) + mu2(jc, ir));
      return div_msf(ld(s.u, ix3(k, jc, iu, ny, nx + 1)) * (c1 * muu_c + c2), g.msfuy, g.rmsfuy, ix2(jc, iu, nx + 1));
    };
    auto rwq = [&](int kf, int jc) {
      return ld(s.w, ix3(kf, jc, i, ny, nx)) * (ld(g.c1f, kf) * mu2(jc, i) + ld(g.c2f, kf)) /
             ld(g.msfty, ix2(jc, i, nx));
    };
    const double f_v = 0.5 * (ld(g.f, ix2(sj, i, nx)) + ld(g.f, ix2(nj, i, nx)));
    const double e_v = 0.5 * (ld(g.e, ix2(sj, i, nx)) + ld(g.e, ix2(nj, i, nx)));
    const double sina_v = 0.5 * (ld(g.sina, ix2(sj, i, nx)) + ld(g.sina, ix2(nj, i, nx)));
    const double msf_v = div_msf(ld(g.msfvy, ix2(j, i, nx)), g.msfvx, g.rmsfvx, ix2(j, i, nx));
    double rv_cor;
    if (f_v != 0.0 || e_v != 0.0) {
      const double ru_quad = 0.25 * (ruq(sj, i) + ruq(sj, i + 1) + ruq(nj, i) + ruq(nj, i + 1));
      rv_cor = -msf_v * f_v * ru_quad;
      const double rw_quad = 0.25 * (rwq(k, sj) + rwq(k + 1, sj) + rwq(k, nj) + rwq(k + 1, nj));
      rv_cor = rv_cor + msf_v * e_v * sina_v * rw_quad;
    } else {
      rv_cor = -msf_v * f_v * 0.0;
      rv_cor = rv_cor + msf_v * e_v * sina_v * 0.0;
    }
    if (run_boundary && (j == 0 || j == ny)) rv_cor = rv_cor * 0.0;
    v_t = v_t + rv_cor;
  }
  o.v_tend[cv] = v_t;
  const size_t f2 = ix2(j, i, nx);
  const double mass_ref = c1 * ld(muvs, f2) + c2;
  const double mass_cur = c1 * ld(muv, f2) + c2;
  o.v_w[cv] = div_msf(mass_ref * ld(ref.v, cv) - mass_cur * ld(s.v, cv), g.msfvx, g.rmsfvx, f2);
}

// ---------------------------------------------------------------------------
// Order<=6 horizontal phi advection sums of rhs_ph under specified lateral BCs
// (core/rhs_ph.py:87-173) at mass cell (j, i) of one face level.  PT(dr, dc)
// is phi_total at (j+dr, i+dc) (|dr|, |dc| <= 3, read only where the row and
// column masks select), FY(jv) / FX(iu) the mass-weighted v / u face flows.
// y: 6th order on rows 3..ny-4, 4th order on rows 2 and ny-3, 2nd order on
// rows 1 and ny-2, none on rows 0 and ny-1; x: 6th order on columns 3..nx-4,
// 2nd order on columns 1 and nx-2, none elsewhere.  The masked branches are
// summed like the reference's where-terms.
// ---------------------------------------------------------------------------
template <typename PTF, typename FYF, typename FXF>
__device__ __forceinline__ void ph_adv_order6(int j, int i, int ny, int nx, PTF PT, FYF FY, FXF FX, double &adv_y,
                                              double &adv_x) {
  double y6 = 0.0, y4 = 0.0, y2 = 0.0;
  if (j >= 3 && j <= ny - 4) {
    const double d1 = PT(1, 0) - PT(-1, 0), d2 = PT(2, 0) - PT(-2, 0), d3 = PT(3, 0) - PT(-3, 0);
    y6 = (FY(j + 1) + FY(j)) * div_rcp(45.0 * d1 - 9.0 * d2 + d3, 60.0, R60);
  }
  if (j == 2 || j == ny - 3) {
    const double d1 = PT(1, 0) - PT(-1, 0), d2 = PT(2, 0) - PT(-2, 0);
    y4 = (FY(j + 1) + FY(j)) * div_rcp(8.0 * d1 - d2, 12.0, R12);
  }
  if (j == 1 || j == ny - 2) {
    const double a0 = PT(0, 0);
    y2 = FY(j + 1) * (PT(1, 0) - a0) + FY(j) * (a0 - PT(-1, 0));
  }
  adv_y = (y6 + y4) + y2;
  double x6 = 0.0, x2 = 0.0;
  if (i >= 3 && i <= nx - 4) {
    const double d1 = PT(0, 1) - PT(0, -1), d2 = PT(0, 2) - PT(0, -2), d3 = PT(0, 3) - PT(0, -3);
    x6 = (FX(i + 1) + FX(i)) * div_rcp(45.0 * d1 - 9.0 * d2 + d3, 60.0, R60);
  }
  if (i == 1 || i == nx - 2) {
    const double a0 = PT(0, 0);
    x2 = FX(i + 1) * (PT(0, 1) - a0) + FX(i) * (a0 - PT(0, -1));
  }
  adv_x = x6 + x2;
}

// ---------------------------------------------------------------------------
// w faces, tiled: w advection and rhs_ph horizontal stencils from tiles.
// ORD6 selects rhs_ph's order<=6 specified-boundary horizontal advection
// (h_sca_adv_order >= 4 with specified lateral BCs), otherwise order 2.
// ---------------------------------------------------------------------------
template <typename F, bool ORD6, bool DEG>
__global__ void __launch_bounds__(TSX *TSY, WG_WFACE_MINB) k_wface_tiled(Grid g, StateR s, StateR ref, const double *ru,
                                                           const double *rv, const double *rom,
                                                           const double *ww_stage, const double *qtot,
                                                           const double *mub, const double *mut, const double *muts0,
                                                           const double *muu, const double *muv,
                                                           const double *base_w, int top_lid, int moist_cqw,
                                                           int w_coriolis, WFaceOut o, PhysW pw) {
  constexpr bool deg = DEG;  // the specified-boundary advection degradation
  using TQ = Tile<3, 3>;
  using TR = Tile<1, 0>;
  using TV = Tile<0, 1>;
  constexpr int PHH = ORD6 ? 3 : 1;  // halo of the phi_total tile
  using TP = Tile<PHH, PHH>;
  __shared__ double sw[TQ::N];
  __shared__ double sru[TR::N];
  __shared__ double srv[TV::N];
  __shared__ double spt[TP::N];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * TSX, j0 = blockIdx.y * TSY, k = blockIdx.z;
  const int i = i0 + tx, j = j0 + ty;
  const size_t pm = (size_t)ny * nx;
  load_tile<3, 3>(sw, s.w + (size_t)k * pm, nx, i0, j0, nx, ny, 0.0);
  // ru / rv interpolated to the full level k (flux_advection.py:1332-1352)
  {
    const int kh = (k == nz) ? nz - 1 : k;
    for (int e = ty * TSX + tx; e < TR::N; e += TSX * TSY) {
      const int r = e / TR::W, cc = e - r * TR::W;
      const int jj = wrp(j0 + r, ny), ii = wrp(i0 - 1 + cc, nx);
      double val;
      if (k == 0 || k == nz) {
        val = ld(ru, ix3(kh, jj, ii, ny, nx));
      } else {
        val = ld(g.fnm, k) * ld(ru, ix3(k, jj, ii, ny, nx)) + ld(g.fnp, k) * ld(ru, ix3(k - 1, jj, ii, ny, nx));
      }
      sru[e] = val;
    }
    for (int e = ty * TSX + tx; e < TV::N; e += TSX * TSY) {
      const int r = e / TV::W, cc = e - r * TV::W;
      const int jj = wrp(j0 - 1 + r, ny), ii = wrp(i0 + cc, nx);
      double val;
      if (k == 0 || k == nz) {
        val = ld(rv, ix3(kh, jj, ii, ny, nx));
      } else {
        val = ld(g.fnm, k) * ld(rv, ix3(k, jj, ii, ny, nx)) + ld(g.fnp, k) * ld(rv, ix3(k - 1, jj, ii, ny, nx));
      }
      srv[e] = val;
    }
    for (int e = ty * TSX + tx; e < TP::N; e += TSX * TSY) {
      const int r = e / TP::W, cc = e - r * TP::W;
      const size_t q = (size_t)k * pm + (size_t)wrp(j0 - PHH + r, ny) * nx + wrp(i0 - PHH + cc, nx);
      const double p = ld(s.ph_pert, q);
      spt[e] = p + (ld(s.ph_total, q) - p);
    }
  }
  __syncthreads();
  if (i >= nx || j >= ny) return;
  const size_t cw = ix3(k, j, i, ny, nx);
  const size_t c2d = ix2(j, i, nx);
  auto W_ = [&](int r, int cc) { return sw[(r + 3) * TQ::W + (cc + 3)]; };
  const double msftx = ld(g.msftx, c2d);
  auto fqx = [&](int m) {
    const double vel = sru[ty * TR::W + (m + 1)];
    if (deg)
      return hflux_spec<F>(i0 + m, nx, false, vel, W_(ty, m - 3), W_(ty, m - 2), W_(ty, m - 1), W_(ty, m),
                           W_(ty, m + 1), W_(ty, m + 2));
    return hflux5<F>(vel, W_(ty, m - 3), W_(ty, m - 2), W_(ty, m - 1), W_(ty, m), W_(ty, m + 1), W_(ty, m + 2));
  };
  // the specified degradation: tiered faces and no horizontal divergence on
  // the outermost cells (flux_advection.py:1305-1318)
  const bool xin = !deg || (i >= 1 && i <= nx - 2), yin = !deg || (j >= 1 && j <= ny - 2);
  double adv = -msftx * g.rdx * (xin ? (fqx(tx + 1) - fqx(tx)) : 0.0);
  if (ny > 1 || deg) {
    auto fqy = [&](int r) {
      const double vel = srv[(r + 1) * TV::W + tx];
      if (deg)
        return hflux_spec<F>(j0 + r, ny, false, vel, W_(r - 3, tx), W_(r - 2, tx), W_(r - 1, tx), W_(r, tx),
                             W_(r + 1, tx), W_(r + 2, tx));
      return hflux5<F>(vel, W_(r - 3, tx), W_(r - 2, tx), W_(r - 1, tx), W_(r, tx), W_(r + 1, tx), W_(r + 2, tx));
    };
    adv = adv - msftx * g.rdy * (yin ? (fqy(ty + 1) - fqy(ty)) : 0.0);
  }
  {
    auto wc = [&](int kk) { return ld(s.w, ix3(kk, j, i, ny, nx)); };
    auto velf = [&](int m) { return 0.5 * (ld(rom, ix3(m, j, i, ny, nx)) + ld(rom, ix3(m - 1, j, i, ny, nx))); };
    auto vfw = [&](int m) {
      if (m <= 0) return 0.0;
      if (m == 1) return velf(1) * 0.5 * (wc(1) + wc(0));
      if (m < nz) return vflux3<F>(velf(m), wc(m - 2), wc(m - 1), wc(m), wc(m + 1));
      if (m == nz && !top_lid) return velf(nz) * 0.5 * (wc(nz) + wc(nz - 1));
      return 0.0;
    };
    double vt = 0.0;
    if (k >= 1 && k <= nz - 1) vt = -ld(g.rdn, k) * (vfw(k + 1) - vfw(k));
    if (k == nz && !top_lid) vt = 0.0 + 2.0 * ld(g.rdn, nz - 1) * vfw(nz);
    adv = adv + vt;
  }
  double w_t;
  if (base_w != nullptr) {
    const double mass_f = ld(g.c1f, k) * ld(s.mu_total, c2d) + ld(g.c2f, k);
    w_t = ld(base_w, cw) * mass_f + adv;
  } else {
    w_t = adv;
  }
  if (pw.rw_tendf != nullptr || (pw.rk1 && pw.w_save != nullptr)) {
    // rk_addtend_dry (rk_addtend_dry.py:490-546): w += (rw_tendf + [rk1] w_save msfty) / msfty
    double r = (pw.rw_tendf != nullptr) ? ld(pw.rw_tendf, cw) : 0.0;
    if (pw.rk1 && pw.w_save != nullptr) r = r + ld(pw.w_save, cw) * ld(g.msfty, c2d);
    w_t = w_t + div_msf(r, g.msfty, g.rmsfty, c2d);
  }
  const double mub_c = ld(mub, c2d), mut_c = ld(mut, c2d);
  const double mu_prime = mut_c - mub_c;
  const double minv = ld(g.rmsfty, c2d);  // == 1.0 / msfty
  auto Pp = [&](int kk) { return ld(s.p_pert, ix3(kk, j, i, ny, nx)); };
  auto Qt = [&](int kk) { return ld(qtot, ix3(kk, j, i, ny, nx)); };
  double rw = 0.0, cqw = 0.0;
  if (k >= 1 && k <= nz - 1) {
    if (moist_cqw) {
      const double ci = 0.5 * (Qt(k) + Qt(k - 1));
      const double cq1 = 1.0 / (1.0 + ci);
      const double cq2 = ci * cq1;
      rw = minv * G * (cq1 * ld(g.rdn, k) * (Pp(k) - Pp(k - 1)) - ld(g.c1f, k) * mu_prime -
                       cq2 * (ld(g.c1f, k) * mub_c + ld(g.c2f, k)));
      cqw = cq1;
    } else {
      rw = minv * G * (ld(g.rdn, k) * (Pp(k) - Pp(k - 1)) - ld(g.c1f, k) * mu_prime);
      cqw = 1.0;
    }
  } else if (k == nz) {
    if (moist_cqw) {
      const double ct = 0.5 * (Qt(nz - 1) + Qt(nz - 2));
      const double c1t = 1.0 / (1.0 + ct);
      const double c2t = ct * c1t;
      rw = minv * G * (c1t * 2.0 * ld(g.rdnw, nz - 1) * (-Pp(nz - 1)) - ld(g.c1f, nz) * mu_prime -
                       c2t * (ld(g.c1f, nz) * mub_c + ld(g.c2f, nz)));
    } else {
      rw = minv * G * (2.0 * ld(g.rdnw, nz - 1) * (-Pp(nz - 1)) - ld(g.c1f, nz) * mu_prime);
    }
  }
  rw = rw + w_t;
  if (w_coriolis && k >= 1 && k <= nz - 1) {
    const double muu_i = ld(muu, ix2(j, i, nx + 1)), muu_ip = ld(muu, ix2(j, i + 1, nx + 1));
    const double muv_j = ld(muv, ix2(j, i, nx)), muv_jp = ld(muv, ix2(j + 1, i, nx));
    const double fuy_i = ld(g.msfuy, ix2(j, i, nx + 1)), fuy_ip = ld(g.msfuy, ix2(j, i + 1, nx + 1));
    const double fvx_j = ld(g.msfvx, ix2(j, i, nx)), fvx_jp = ld(g.msfvx, ix2(j + 1, i, nx));
    const double rfuy_i = ld(g.rmsfuy, ix2(j, i, nx + 1)), rfuy_ip = ld(g.rmsfuy, ix2(j, i + 1, nx + 1));
    const double rfvx_j = ld(g.rmsfvx, ix2(j, i, nx)), rfvx_jp = ld(g.rmsfvx, ix2(j + 1, i, nx));
    auto lev = [&](int kk, double &ru_m, double &u_m, double &rv_m, double &v_m) {
      const double c1 = ld(g.c1h, kk), c2 = ld(g.c2h, kk);
      const double u0 = ld(s.u, ix3(kk, j, i, ny, nx + 1)), u1 = ld(s.u, ix3(kk, j, i + 1, ny, nx + 1));
      const double v0 = ld(s.v, ix3(kk, j, i, ny + 1, nx)), v1 = ld(s.v, ix3(kk, j + 1, i, ny + 1, nx));
      const double rs0 = div_rcp((c1 * muu_i + c2) * u0, fuy_i, rfuy_i);
      const double rs1 = div_rcp((c1 * muu_ip + c2) * u1, fuy_ip, rfuy_ip);
      const double vs0 = div_rcp((c1 * muv_j + c2) * v0, fvx_j, rfvx_j);
      const double vs1 = div_rcp((c1 * muv_jp + c2) * v1, fvx_jp, rfvx_jp);
      ru_m = 0.5 * (rs0 + rs1);
      u_m = 0.5 * (u0 + u1);
      rv_m = 0.5 * (vs0 + vs1);
      v_m = 0.5 * (v0 + v1);
    };
    double ru_a, u_a, rv_a, v_a, ru_b, u_b, rv_b, v_b;
    lev(k, ru_a, u_a, rv_a, v_a);
    lev(k - 1, ru_b, u_b, rv_b, v_b);
    const double fm = ld(g.fnm, k), fp = ld(g.fnp, k);
    const double ru_f = fm * ru_a + fp * ru_b, u_f = fm * u_a + fp * u_b;
    const double rv_f = fm * rv_a + fp * rv_b, v_f = fm * v_a + fp * v_b;
    const double mxy = div_msf(ld(g.msftx, c2d), g.msfty, g.rmsfty, c2d);
    const double cor = ld(g.e, c2d) * (ld(g.cosa, c2d) * ru_f - mxy * ld(g.sina, c2d) * rv_f);
    const double curv = W_RERADIUS * (ru_f * u_f + mxy * rv_f * v_f);
    rw = rw + (cor + curv);
  }
  o.rw_tend[cw] = rw;
  o.cqw[cw] = cqw;
  {
    auto PT = [&](int r, int cc) { return spt[(r + PHH) * TP::W + (cc + PHH)]; };
    auto pht = [&](int kk) {  // column value at level kk
      const size_t q = ix3(kk, j, i, ny, nx);
      const double p = ld(s.ph_pert, q);
      return p + (ld(s.ph_total, q) - p);
    };
    double out = 0.0;
    if (k >= 1 && k <= nz - 1) {
      auto wdwn = [&](int m) {
        const double wwm = 0.5 * (ld(ww_stage, ix3(m + 1, j, i, ny, nx)) + ld(ww_stage, ix3(m, j, i, ny, nx)));
        return wwm * ld(g.rdnw, m) * (pht(m + 1) - pht(m));
      };
      const double term3 = ld(g.fnm, k) * wdwn(k) + ld(g.fnp, k) * wdwn(k - 1);
      out = 0.0 + (-term3);
      const double mass_f = ld(g.c1f, k) * mut_c + ld(g.c2f, k);
      out = out + mass_f * G * ld(s.w, cw) * minv;
      const double c1f = ld(g.c1f, k), c2f = ld(g.c2f, k);
      auto vpair = [&](int jv) { return ld(s.v, ix3(k, jv, i, ny + 1, nx)) + ld(s.v, ix3(k - 1, jv, i, ny + 1, nx)); };
      auto muvf = [&](int jv) { return c1f * ld(muv, ix2(jv, i, nx)) + c2f; };
      auto upair = [&](int iu) { return ld(s.u, ix3(k, j, iu, ny, nx + 1)) + ld(s.u, ix3(k - 1, j, iu, ny, nx + 1)); };
      auto muuf = [&](int iu) { return c1f * ld(muu, ix2(j, iu, nx + 1)) + c2f; };
      if constexpr (ORD6) {
        auto FY = [&](int jv) { return muvf(jv) * vpair(jv) * ld(g.msfvy, ix2(jv, i, nx)); };
        auto FX = [&](int iu) { return muuf(iu) * upair(iu) * ld(g.msfux, ix2(j, iu, nx + 1)); };
        auto PTo = [&](int dr, int dc) { return PT(ty + dr, tx + dc); };
        double adv_y, adv_x;
        ph_adv_order6(j, i, ny, nx, PTo, FY, FX, adv_y, adv_x);
        const double msfty_c = ld(g.msfty, c2d);
        const double adv = div_rcp(0.25 * g.rdy, msfty_c, minv) * adv_y + div_rcp(0.25 * g.rdx, msfty_c, minv) * adv_x;
        out = out + (-adv);
      } else {
        const double pti = PT(ty, tx);
        const double dn_ = PT(ty + 1, tx) - pti;
        const double ds_ = pti - PT(ty - 1, tx);
        const double flux_y = muvf(j + 1) * vpair(j + 1) * dn_ + muvf(j) * vpair(j) * ds_;
        out = out + (-(0.25 * g.rdy * minv)) * flux_y;
        const double de_ = PT(ty, tx + 1) - pti;
        const double dw_ = pti - PT(ty, tx - 1);
        const double flux_x = muuf(i + 1) * upair(i + 1) * de_ + muuf(i) * upair(i) * dw_;
        out = out + (-(0.25 * g.rdx * minv)) * flux_x;
      }
    } else if (k == nz && !top_lid) {
      const double mass_f = ld(g.c1f, nz) * mut_c + ld(g.c2f, nz);
      out = mass_f * G * ld(s.w, cw) * minv;
      if constexpr (ORD6) {
        // open-top face row: winds extrapolated with cfn/cfn1, weight 0.5
        // (core/rhs_ph.py:290-343)
        const double c1t = ld(g.c1f, nz), c2t = ld(g.c2f, nz);
        auto FY = [&](int jv) {
          const double vt = g.cfn * ld(s.v, ix3(nz - 1, jv, i, ny + 1, nx)) + g.cfn1 * ld(s.v, ix3(nz - 2, jv, i, ny + 1, nx));
          return (c1t * ld(muv, ix2(jv, i, nx)) + c2t) * vt * ld(g.msfvy, ix2(jv, i, nx));
        };
        auto FX = [&](int iu) {
          const double ut = g.cfn * ld(s.u, ix3(nz - 1, j, iu, ny, nx + 1)) + g.cfn1 * ld(s.u, ix3(nz - 2, j, iu, ny, nx + 1));
          return (c1t * ld(muu, ix2(j, iu, nx + 1)) + c2t) * ut * ld(g.msfux, ix2(j, iu, nx + 1));
        };
        auto PTo = [&](int dr, int dc) { return PT(ty + dr, tx + dc); };
        double adv_y, adv_x;
        ph_adv_order6(j, i, ny, nx, PTo, FY, FX, adv_y, adv_x);
        const double msfty_c = ld(g.msfty, c2d);
        out = out + ((-div_rcp(0.5 * g.rdy, msfty_c, minv)) * adv_y - div_rcp(0.5 * g.rdx, msfty_c, minv) * adv_x);
      }
    }
    o.ph_tend[cw] = out;
  }
  const double mass_f_ref = ld(g.c1f, k) * ld(muts0, c2d) + ld(g.c2f, k);
  const double mass_f_cur = ld(g.c1f, k) * mut_c + ld(g.c2f, k);
  o.w_w[cw] = div_msf(mass_f_ref * ld(ref.w, cw) - mass_f_cur * ld(s.w, cw), g.msfty, g.rmsfty, c2d);
  const double php = ld(s.ph_pert, cw);
  o.ph_w[cw] = ld(ref.ph_pert, cw) - php;
  o.pt1[cw] = ld(ref.ph_pert, cw) + (ld(s.ph_total, cw) - php);
  o.ww[cw] = ld(ww_stage, cw);
  if (k == 0) o.phb0[c2d] = ld(s.ph_total, cw) - php;
}

// ---------------------------------------------------------------------------
// Transport velocities (flux_advection.py:394-470) and the specified stage
// omega (flux_advection.py:180-232), level-parallel: a block owns 32 columns,
// its warps split the levels, and the column sum / cumulative sum run serially
// per column out of shared memory (same order as the reference).
// ---------------------------------------------------------------------------
inline size_t transport_smem_bytes(int nz) { return (size_t)2 * nz * 32 * sizeof(double); }

#ifdef WG_TRANSPORT_MINB
#define WG_TRANSPORT_BOUNDS __launch_bounds__(256, WG_TRANSPORT_MINB)
#else
#define WG_TRANSPORT_BOUNDS __launch_bounds__(256)
#endif
__global__ void WG_TRANSPORT_BOUNDS k_transport_tiled(Grid g, const double *u, const double *v,
                                                          const double *mu_total, double *ru, double *rv, double *rom,
                                                          double *ww_spec) {
  extern __shared__ double sm[];
  const int tx = threadIdx.x, ty = threadIdx.y;  // blockDim (32, 8)
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = blockIdx.x * 32 + tx, j = blockIdx.y;
  const bool valid = i < nx;
  auto D0 = [&](int k) -> double & { return sm[(size_t)k * 32 + tx]; };
  auto D1 = [&](int k) -> double & { return sm[(size_t)(nz + k) * 32 + tx]; };
  int ip = 0, im = 0, jp = 0, jm = 0;
  double mu_c = 0, muu_i = 0, muu_ip = 0, muv_j = 0, muv_jp = 0, msfuy_i = 1, msfuy_ip = 1, msfvx_j = 1, msfvx_jp = 1,
         msftx = 1;
  double muu_s_i = 0, muu_s_ip = 0, muv_s_j = 0, muv_s_jp = 0, fuy_ip = 1, fvx_jp = 1;
  double rmsfuy_i = 1, rmsfuy_ip = 1, rmsfvx_j = 1, rmsfvx_jp = 1, rfuy_ip = 1, rfvx_jp = 1;
  if (valid) {
    ip = wrp(i + 1, nx); im = wrp(i - 1, nx); jp = wrp(j + 1, ny); jm = wrp(j - 1, ny);
    mu_c = ld(mu_total, ix2(j, i, nx));
    muu_i = 0.5 * (mu_c + ld(mu_total, ix2(j, im, nx)));
    muu_ip = 0.5 * (ld(mu_total, ix2(j, ip, nx)) + mu_c);
    muv_j = 0.5 * (mu_c + ld(mu_total, ix2(jm, i, nx)));
    muv_jp = 0.5 * (ld(mu_total, ix2(jp, i, nx)) + mu_c);
    msfuy_i = ld(g.msfuy, ix2(j, i, nx + 1)); msfuy_ip = ld(g.msfuy, ix2(j, ip, nx + 1));
    msfvx_j = ld(g.msfvx, ix2(j, i, nx)); msfvx_jp = ld(g.msfvx, ix2(jp, i, nx));
    rmsfuy_i = ld(g.rmsfuy, ix2(j, i, nx + 1)); rmsfuy_ip = ld(g.rmsfuy, ix2(j, ip, nx + 1));
    rmsfvx_j = ld(g.rmsfvx, ix2(j, i, nx)); rmsfvx_jp = ld(g.rmsfvx, ix2(jp, i, nx));
    msftx = ld(g.msftx, ix2(j, i, nx));
    if (ww_spec != nullptr) {
      const double mu_w = (i == 0) ? mu_c : ld(mu_total, ix2(j, i - 1, nx));
      muu_s_i = 0.5 * (mu_c + mu_w);
      muu_s_ip = (i + 1 == nx) ? mu_c : 0.5 * (ld(mu_total, ix2(j, i + 1, nx)) + mu_c);
      const double mu_s = (j == 0) ? mu_c : ld(mu_total, ix2(j - 1, i, nx));
      muv_s_j = 0.5 * (mu_c + mu_s);
      muv_s_jp = (j + 1 == ny) ? mu_c : 0.5 * (ld(mu_total, ix2(j + 1, i, nx)) + mu_c);
      fuy_ip = ld(g.msfuy, ix2(j, i + 1, nx + 1));
      fvx_jp = ld(g.msfvx, ix2(j + 1, i, nx));
      rfuy_ip = ld(g.rmsfuy, ix2(j, i + 1, nx + 1));
      rfvx_jp = ld(g.rmsfvx, ix2(j + 1, i, nx));
    }
  }
  if (valid) {
    for (int k = ty; k < nz; k += 8) {
      const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
      const double u_i = ld(u, ix3(k, j, i, ny, nx + 1)), v_j = ld(v, ix3(k, j, i, ny + 1, nx));
      const double ru_i = div_rcp((c1 * muu_i + c2) * u_i, msfuy_i, rmsfuy_i);
      const double ru_ip = div_rcp((c1 * muu_ip + c2) * ld(u, ix3(k, j, ip, ny, nx + 1)), msfuy_ip, rmsfuy_ip);
      const double rv_j = div_rcp((c1 * muv_j + c2) * v_j, msfvx_j, rmsfvx_j);
      const double rv_jp = div_rcp((c1 * muv_jp + c2) * ld(v, ix3(k, jp, i, ny + 1, nx)), msfvx_jp, rmsfvx_jp);
      D0(k) = ld(g.dnw, k) * msftx * (g.rdx * (ru_ip - ru_i) + g.rdy * (rv_jp - rv_j));
      ru[ix3(k, j, i, ny, nx)] = ru_i;
      rv[ix3(k, j, i, ny, nx)] = rv_j;
      if (ww_spec != nullptr) {
        const double a0 = div_rcp((c1 * muu_s_i + c2) * u_i, msfuy_i, rmsfuy_i);
        const double a1 = div_rcp((c1 * muu_s_ip + c2) * ld(u, ix3(k, j, i + 1, ny, nx + 1)), fuy_ip, rfuy_ip);
        const double b0 = div_rcp((c1 * muv_s_j + c2) * v_j, msfvx_j, rmsfvx_j);
        const double b1 = div_rcp((c1 * muv_s_jp + c2) * ld(v, ix3(k, j + 1, i, ny + 1, nx)), fvx_jp, rfvx_jp);
        D1(k) = msftx * ld(g.dnw, k) * (g.rdx * (a1 - a0) + g.rdy * (b1 - b0));
      }
    }
  }
  __syncthreads();
  // Column sums (serial chains over shared memory, loads batched ahead of
  // the adds), then the level-parallel increments, the serial prefix sum in
  // place, and the level-parallel stores.  Thread row 0 does rom, row 1 the
  // specified stage omega.
  __shared__ double s_dm[2][32];
  auto serial_sum = [&](auto D) {
    constexpr int SU = 8;
    double acc = D(0);
    int k = 1;
    for (; k + SU <= nz; k += SU) {
      double r[SU];
#pragma unroll
      for (int u = 0; u < SU; ++u) r[u] = D(k + u);
#pragma unroll
      for (int u = 0; u < SU; ++u) acc = acc + r[u];
    }
    for (; k < nz; ++k) acc = acc + D(k);
    return acc;
  };
  auto serial_prefix = [&](auto D) {  // D(k) <- D(0) + ... + D(k) for k < nz - 1
    constexpr int SU = 8;
    double cum = D(0);
    int k = 1;
    for (; k + SU <= nz - 1; k += SU) {
      double r[SU];
#pragma unroll
      for (int u = 0; u < SU; ++u) r[u] = D(k + u);
#pragma unroll
      for (int u = 0; u < SU; ++u) {
        cum = cum + r[u];
        D(k + u) = cum;
      }
    }
    for (; k < nz - 1; ++k) {
      cum = cum + D(k);
      D(k) = cum;
    }
  };
  const bool spec = ww_spec != nullptr;
  if (valid && ty == 0) s_dm[0][tx] = serial_sum(D0);
  if (valid && ty == 1 && spec) s_dm[1][tx] = serial_sum(D1);
  __syncthreads();
  if (valid) {
    const double dmdt = s_dm[0][tx];
    const double dm = spec ? s_dm[1][tx] : 0.0;
    for (int k = ty; k < nz - 1; k += 8) {
      const double dc = ld(g.dnw, k) * ld(g.c1h, k);
      D0(k) = -(dc * dmdt) - D0(k);
      if (spec) D1(k) = -(dc * dm) - D1(k);
    }
  }
  __syncthreads();
  if (valid && ty == 0) serial_prefix(D0);
  if (valid && ty == 1 && spec) serial_prefix(D1);
  __syncthreads();
  if (valid) {
    for (int f = ty; f <= nz; f += 8) {
      const double rv_ = (f >= 1 && f <= nz - 1) ? D0(f - 1) : 0.0;
      rom[ix3(f, j, i, ny, nx)] = rv_;
      if (spec) ww_spec[ix3(f, j, i, ny, nx)] = (f >= 1 && f <= nz - 1) ? D1(f - 1) : 0.0;
    }
  }
}

}  // namespace wg
