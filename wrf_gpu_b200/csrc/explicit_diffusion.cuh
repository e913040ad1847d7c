// Second-order explicit diffusion closures of the RK stage, added to the
// stage's coupled u, v, w, theta tendencies after the 6th-order filter
// (operational_mode.py:2878-2960):
//
//  * diff_opt = 1, km_opt = 4: WRF's 2-D Smagorinsky horizontal diffusion on
//    coordinate surfaces, the real-data default.  k_smag_km forms the eddy
//    viscosity xkmh on mass cells from the horizontal deformation of the stage
//    (u, v) (horizontal_deformation_2d + smag2d_horizontal_km,
//    dynamics/explicit_diffusion.py:960-1212, called without metrics, so the
//    map factors are one and the slope terms vanish); k_smag_apply adds
//    d/dx(mass_f K_f d./dx) + d/dy(...) of every field on its own stagger
//    (_hdiff_coord_scalar, :1233-1284; theta as the perturbation from 300 K
//    with xkhh = xkmh / prandtl, momentum with xkmh, w with xkmh averaged to
//    the w levels, :1215-1230, 1287-1365).
//  * const_nu_m2_s > 0: constant-K diffusion in the mass-conservative flux
//    form (conservative_constant_k_diffusion_tendency, :282-331) on u, v, w
//    and theta, horizontal plus vertical with the stage's mean layer depth
//    dz = max(mean(diff(ph_total) / g), 1) (operational_mode.py:2757-2758),
//    reduced on the device in a fixed order (k_dz_partial / k_dz_final).
//
// Every neighbour is taken with the reference's periodic roll over the
// array's own extent (the core mass extent for the Smagorinsky fields, whose
// u / v wrap faces repeat face 0; the full staggered extent for constant K),
// whatever the lateral boundary type, as the reference's jnp.roll does.
#pragma once
#include "dycore_common.cuh"

namespace wg {

constexpr double PRANDTL = 1.0 / 3.0;  // explicit_diffusion.py:956
constexpr double RPRANDTL = 1.0 / PRANDTL;  // its correctly rounded reciprocal, for div_rcp

__device__ __forceinline__ int roll_idx(int q, int n) { return q < 0 ? q + n : (q >= n ? q - n : q); }

struct DiffArgs {
  const double *u, *v, *w, *theta, *mu;  // the stage state (mu = mu_total)
  double *u_tend, *v_tend, *w_tend, *t_tend;
  const double *xkmh;                    // Smagorinsky: eddy viscosity on mass cells
  double c_s;
  double nu;                             // constant K (m^2/s)
  const double *dz;                      // constant K: device scalar, the mean layer depth
};

// ---------------------------------------------------------------------------
// Smagorinsky eddy viscosity (mass cells): index space (nx, ny, nz).
// ---------------------------------------------------------------------------
__global__ void k_smag_km(Grid g, DiffArgs a, double *xkmh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny;
  if (i >= nx || j >= ny) return;
  const int nxu = nx + 1;
  auto U = [&](int jj, int ii) { return ld(a.u, ix3(k, jj, ii, ny, nxu)); };  // core u: ii < nx
  auto V = [&](int jj, int ii) { return ld(a.v, ix3(k, jj, ii, ny + 1, nx)); };  // core v: jj < ny
  const int ie = roll_idx(i + 1, nx), jn = roll_idx(j + 1, ny);
  // D11 = 2 du/dx, D22 = 2 dv/dy at the cell (explicit_diffusion.py:1033-1057)
  // every x / dx and x / dy is an exact div_rcp with g.rdx = 1/dx, g.rdy = 1/dy
  const double d11 = 2.0 * div_rcp(U(j, ie) - U(j, i), g.dx, g.rdx);
  const double d22 = 2.0 * div_rcp(V(jn, i) - V(j, i), g.dy, g.rdy);
  // D12 = du/dy + dv/dx on the SW corner (ic, jc) of a cell (:1059-1112)
  auto d12 = [&](int jc, int ic) {
    const int js = roll_idx(jc - 1, ny), iw = roll_idx(ic - 1, nx);
    const double dudy = div_rcp(U(jc, ic) - U(js, ic), g.dy, g.rdy);
    const double dvdx = div_rcp(V(jc, ic) - V(jc, iw), g.dx, g.rdx);
    return dudy + dvdx;
  };
  // four-corner average, SW + NW + SE + NE (:1173-1177)
  const double tmp = 0.25 * (d12(j, i) + d12(jn, i) + d12(j, ie) + d12(jn, ie));
  const double def2 = 0.25 * (d11 - d22) * (d11 - d22) + tmp * tmp;
  const double mlen_h = sqrt((g.dx / 1.0) * (g.dy / 1.0));
  double km = a.c_s * a.c_s * mlen_h * mlen_h * sqrt(def2);
  const double cap = 10.0 * mlen_h;
  km = km < cap ? km : cap;  // jnp.minimum (both finite here)
  xkmh[ix3(k, j, i, ny, nx)] = km;
}

// The coordinate-surface flux divergence of one field at one point
// (_hdiff_coord_scalar): F(jj, ii) the field, K(jj, ii) the viscosity,
// Ms(jj, ii) the mass, over a periodic (ny_f, nx_f) plane.
template <typename FF, typename FK, typename FM>
__device__ __forceinline__ double hdiff_point(const Grid &g, int j, int i, int ny_f, int nx_f, FF F, FK K, FM Ms) {
  const int ie = roll_idx(i + 1, nx_f), iw = roll_idx(i - 1, nx_f);
  const double kc = K(j, i), mc = Ms(j, i), fc = F(j, i);
  const double mkrdxp = 0.5 * (K(j, ie) + kc) * (0.5 * (Ms(j, ie) + mc)) * g.rdx;
  const double mkrdxm = 0.5 * (kc + K(j, iw)) * (0.5 * (mc + Ms(j, iw))) * g.rdx;
  double tend = g.rdx * (mkrdxp * (F(j, ie) - fc) - mkrdxm * (fc - F(j, iw)));
  if (ny_f > 1) {
    const int jn = roll_idx(j + 1, ny_f), js = roll_idx(j - 1, ny_f);
    const double mkrdyp = 0.5 * (K(jn, i) + kc) * (0.5 * (Ms(jn, i) + mc)) * g.rdy;
    const double mkrdym = 0.5 * (kc + K(js, i)) * (0.5 * (mc + Ms(js, i))) * g.rdy;
    tend = tend + g.rdy * (mkrdyp * (F(jn, i) - fc) - mkrdym * (fc - F(js, i)));
  }
  return tend;
}

// u-face / v-face dry-air mass weights from the edge-padded face averages of
// mu_total (operational_mode.py:1282-1293, 2769-2772).
__device__ __forceinline__ double mu_u_face(const double *mu, int j, int i, int nx) {
  return i == 0 ? ld(mu, ix2(j, 0, nx))
                : (i == nx ? ld(mu, ix2(j, nx - 1, nx)) : 0.5 * (ld(mu, ix2(j, i - 1, nx)) + ld(mu, ix2(j, i, nx))));
}
__device__ __forceinline__ double mu_v_face(const double *mu, int j, int i, int nx, int ny) {
  return j == 0 ? ld(mu, ix2(0, i, nx))
                : (j == ny ? ld(mu, ix2(ny - 1, i, nx)) : 0.5 * (ld(mu, ix2(j - 1, i, nx)) + ld(mu, ix2(j, i, nx))));
}

// ---------------------------------------------------------------------------
// Smagorinsky tendencies: index space (nx+1, ny+1, nz+1); the u, v, w and
// theta points at (k, j, i), each on its own stagger.
// ---------------------------------------------------------------------------
// 16 resident blocks of 128 per SM (32 registers): 433 x 433 x 50, the
// Smagorinsky pair 1.35 vs 1.58 ms/step unbounded (12: 1.42).
#ifndef WG_SMAG_MINB
#define WG_SMAG_MINB 16
#endif
#if WG_SMAG_MINB > 0
#define WG_SMAG_MINB_BOUNDS __launch_bounds__(128, WG_SMAG_MINB)
#else
#define WG_SMAG_MINB_BOUNDS
#endif
__global__ void WG_SMAG_MINB_BOUNDS k_smag_apply(Grid g, DiffArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxu = nx + 1;
  if (i > nx || j > ny) return;
  const double c1h = k < nz ? ld(g.c1h, k) : 0.0, c2h = k < nz ? ld(g.c2h, k) : 0.0;
  auto KM = [&](int kk, int jj, int ii) { return ld(a.xkmh, ix3(kk, jj, ii, ny, nx)); };
  if (k < nz && j < ny) {
    // u: the core faces 0..nx-1 (face nx repeats face 0)
    const int ic = i == nx ? 0 : i;
    auto F = [&](int jj, int ii) { return ld(a.u, ix3(k, jj, ii, ny, nxu)); };
    auto K = [&](int jj, int ii) { return KM(k, jj, ii); };
    auto Ms = [&](int jj, int ii) { return c1h * mu_u_face(a.mu, jj, ii, nx) + c2h; };
    const size_t c = ix3(k, j, i, ny, nxu);
    a.u_tend[c] = a.u_tend[c] + hdiff_point(g, j, ic, ny, nx, F, K, Ms);
  }
  if (k < nz && i < nx) {
    // v: the core faces 0..ny-1 (face ny repeats face 0)
    const int jc = j == ny ? 0 : j;
    auto F = [&](int jj, int ii) { return ld(a.v, ix3(k, jj, ii, ny + 1, nx)); };
    auto K = [&](int jj, int ii) { return KM(k, jj, ii); };
    auto Ms = [&](int jj, int ii) { return c1h * mu_v_face(a.mu, jj, ii, nx, ny) + c2h; };
    const size_t c = ix3(k, j, i, ny + 1, nx);
    a.v_tend[c] = a.v_tend[c] + hdiff_point(g, jc, i, ny, nx, F, K, Ms);
  }
  if (i < nx && j < ny) {
    // w: xkmh averaged to the w level (bottom / top faces take the nearest level)
    auto KW = [&](int jj, int ii) {
      return k == 0 ? KM(0, jj, ii) : (k == nz ? KM(nz - 1, jj, ii) : 0.5 * (KM(k, jj, ii) + KM(k - 1, jj, ii)));
    };
    auto FW = [&](int jj, int ii) { return ld(a.w, ix3(k, jj, ii, ny, nx)); };
    const double c1f = ld(g.c1f, k), c2f = ld(g.c2f, k);
    auto MF = [&](int jj, int ii) { return c1f * ld(a.mu, ix2(jj, ii, nx)) + c2f; };
    const size_t c = ix3(k, j, i, ny, nx);
    a.w_tend[c] = a.w_tend[c] + hdiff_point(g, j, i, ny, nx, FW, KW, MF);
    if (k < nz) {
      // theta as the perturbation from 300 K, with xkhh = xkmh / prandtl
      auto FT = [&](int jj, int ii) { return ld(a.theta, ix3(k, jj, ii, ny, nx)) - T0; };
      auto KH = [&](int jj, int ii) { return div_rcp(KM(k, jj, ii), PRANDTL, RPRANDTL); };
      auto MH = [&](int jj, int ii) { return c1h * ld(a.mu, ix2(jj, ii, nx)) + c2h; };
      a.t_tend[c] = a.t_tend[c] + hdiff_point(g, j, i, ny, nx, FT, KH, MH);
    }
  }
}

// ---------------------------------------------------------------------------
// Constant K.  The mean layer depth: per row j the sum over (k, i) of
// (ph(k+1) - ph(k)) / g in a fixed order, then one thread sums the rows.
// ---------------------------------------------------------------------------
constexpr int DZ_THREADS = 256;

__global__ void __launch_bounds__(DZ_THREADS) k_dz_partial(Grid g, const double *ph_total, double *partial) {
  __shared__ double s[DZ_THREADS];
  const int j = blockIdx.x;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  double acc = 0.0;
  for (int e = threadIdx.x; e < nz * nx; e += DZ_THREADS) {
    const int k = e / nx, i = e - k * nx;
    acc += div_rcp(ld(ph_total, ix3(k + 1, j, i, ny, nx)) - ld(ph_total, ix3(k, j, i, ny, nx)), G, RG);
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = DZ_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[j] = s[0];
}

__global__ void k_dz_final(Grid g, const double *partial, double *dz) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double sum = 0.0;
  for (int j = 0; j < g.ny; ++j) sum += partial[j];
  const double mean = sum / ((double)g.nz * (double)g.ny * (double)g.nx);
  dz[0] = mean > 1.0 ? mean : 1.0;
}

// One field's constant-K flux divergence at (k, j, i) over its own periodic
// (ny_f, nx_f) extent and nz_f levels (zero flux through the bottom and top).
template <typename FF, typename FM>
__device__ __forceinline__ double constk_point(const Grid &g, int k, int j, int i, int nz_f, int ny_f, int nx_f,
                                               double nu, double dz, double rdz, FF F, FM Ms) {
  const int ie = roll_idx(i + 1, nx_f), iw = roll_idx(i - 1, nx_f);
  const double fc = F(k, j, i), mc = Ms(k, j, i);
  // x fluxes at the faces i+1/2 and i-1/2
  // x / dx, x / dy, x / dz as exact div_rcp (rdz = 1/dz computed once)
  const double fxp = div_rcp(0.5 * (mc + Ms(k, j, ie)) * nu * (F(k, j, ie) - fc), g.dx, g.rdx);
  const double fxm = div_rcp(0.5 * (Ms(k, j, iw) + mc) * nu * (fc - F(k, j, iw)), g.dx, g.rdx);
  double tend = 0.0 + div_rcp(fxp - fxm, g.dx, g.rdx);
  if (ny_f > 1) {
    const int jn = roll_idx(j + 1, ny_f), js = roll_idx(j - 1, ny_f);
    const double fyp = div_rcp(0.5 * (mc + Ms(k, jn, i)) * nu * (F(k, jn, i) - fc), g.dy, g.rdy);
    const double fym = div_rcp(0.5 * (Ms(k, js, i) + mc) * nu * (fc - F(k, js, i)), g.dy, g.rdy);
    tend = tend + div_rcp(fyp - fym, g.dy, g.rdy);
  }
  if (nz_f > 2) {
    const double ftop =
        (k + 1 <= nz_f - 1) ? div_rcp(0.5 * (mc + Ms(k + 1, j, i)) * nu * (F(k + 1, j, i) - fc), dz, rdz) : 0.0;
    const double fbot = (k >= 1) ? div_rcp(0.5 * (Ms(k - 1, j, i) + mc) * nu * (fc - F(k - 1, j, i)), dz, rdz) : 0.0;
    tend = tend + div_rcp(ftop - fbot, dz, rdz);
  }
  return tend;
}

// Index space (nx+1, ny+1, nz+1): u, v, w, theta at (k, j, i) on their own staggers.
// 16 resident blocks of 128 per SM: 433 x 433 x 50, 1.52 vs 1.83 ms/step
// unbounded (12: 1.59).
#ifndef WG_CONSTK_MINB
#define WG_CONSTK_MINB 16
#endif
#if WG_CONSTK_MINB > 0
#define WG_CONSTK_MINB_BOUNDS __launch_bounds__(128, WG_CONSTK_MINB)
#else
#define WG_CONSTK_MINB_BOUNDS
#endif
__global__ void WG_CONSTK_MINB_BOUNDS k_constk_apply(Grid g, DiffArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxu = nx + 1, nyv = ny + 1;
  if (i > nx || j > ny) return;
  const double dz = a.dz[0], nu = a.nu;
  const double rdz = 1.0 / dz;
  if (k < nz && j < ny) {
    auto F = [&](int kk, int jj, int ii) { return ld(a.u, ix3(kk, jj, ii, ny, nxu)); };
    auto Ms = [&](int kk, int jj, int ii) { return ld(g.c1h, kk) * mu_u_face(a.mu, jj, ii, nx) + ld(g.c2h, kk); };
    const size_t c = ix3(k, j, i, ny, nxu);
    a.u_tend[c] = a.u_tend[c] + constk_point(g, k, j, i, nz, ny, nxu, nu, dz, rdz, F, Ms);
  }
  if (k < nz && i < nx) {
    auto F = [&](int kk, int jj, int ii) { return ld(a.v, ix3(kk, jj, ii, nyv, nx)); };
    auto Ms = [&](int kk, int jj, int ii) { return ld(g.c1h, kk) * mu_v_face(a.mu, jj, ii, nx, ny) + ld(g.c2h, kk); };
    const size_t c = ix3(k, j, i, nyv, nx);
    a.v_tend[c] = a.v_tend[c] + constk_point(g, k, j, i, nz, nyv, nx, nu, dz, rdz, F, Ms);
  }
  if (i < nx && j < ny) {
    auto FW = [&](int kk, int jj, int ii) { return ld(a.w, ix3(kk, jj, ii, ny, nx)); };
    auto MF = [&](int kk, int jj, int ii) { return ld(g.c1f, kk) * ld(a.mu, ix2(jj, ii, nx)) + ld(g.c2f, kk); };
    const size_t c = ix3(k, j, i, ny, nx);
    a.w_tend[c] = a.w_tend[c] + constk_point(g, k, j, i, nz + 1, ny, nx, nu, dz, rdz, FW, MF);
    if (k < nz) {
      auto FT = [&](int kk, int jj, int ii) { return ld(a.theta, ix3(kk, jj, ii, ny, nx)); };
      auto MH = [&](int kk, int jj, int ii) { return ld(g.c1h, kk) * ld(a.mu, ix2(jj, ii, nx)) + ld(g.c2h, kk); };
      a.t_tend[c] = a.t_tend[c] + constk_point(g, k, j, i, nz, ny, nx, nu, dz, rdz, FT, MH);
    }
  }
}

}  // namespace wg
