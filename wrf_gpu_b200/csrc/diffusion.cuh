// The 6th-order numerical diffusion filter (diff_6th_opt;
// sixth_order_diffusion_tendency, dynamics/explicit_diffusion.py:160-226),
// added to the stage's coupled u, v, w and theta tendencies
// (operational_mode.py:2870-2876): per field, per horizontal axis, Xue's
// 6th-order fluxes at the cell's two faces
//   p0 = 10 (f_i - f_i-1) - 5 (f_i+1 - f_i-2) + (f_i+2 - f_i-3),  p1 = p0 shifted by +1,
// zeroed where they point up-gradient (the monotonic form the stage uses),
// coef (p1 - p0) with coef = diff_6th_factor * 0.015625 / (2 dt), x then y
// (y only on fields with more than one row); neighbours wrap around the
// field's own extent (the reference rolls each staggered array), and the
// sum is coupled by the field's dry-air mass (mass_u / mass_v from the
// edge-padded face averages of mu_total, mass_h, mass_f).
#pragma once
#include "dycore_common.cuh"

namespace wg {

struct Diff6Args {
  const double *u, *v, *w, *theta, *mu;  // the stage state
  double *u_tend, *v_tend, *w_tend, *t_tend;
  double coef;
};

constexpr int D6_TX = 32, D6_TY = 8, D6_H = 3;
constexpr int D6_W = D6_TX + 2 * D6_H, D6_R = D6_TY + 2 * D6_H;

// q in [-3, n + 2] wrapped into [0, n) (one correction when n >= 3); tile
// entries beyond that range are never read by a valid cell and are clamped.
__device__ __forceinline__ int wrap(int q, int n) {
  if (n < 3) return q < 0 ? q + n * ((-q + n - 1) / n) : q % n;
  q = q < 0 ? q + n : (q >= n ? q - n : q);
  return q < n ? q : n - 1;
}

// One axis of the filter from 7 consecutive values f[-3..3] (f[0] the cell).
__device__ __forceinline__ double sixth_1d(const double *f, int stride, double coef) {
  const double fm3 = f[-3 * stride], fm2 = f[-2 * stride], fm1 = f[-stride], f0 = f[0], fp1 = f[stride],
               fp2 = f[2 * stride], fp3 = f[3 * stride];
  double p0 = 10.0 * (f0 - fm1) - 5.0 * (fp1 - fm2) + (fp2 - fm3);
  double p1 = 10.0 * (fp1 - f0) - 5.0 * (fp2 - fm1) + (fp3 - fm2);
  if (p0 * (f0 - fm1) <= 0.0) p0 = 0.0;
  if (p1 * (fp1 - f0) <= 0.0) p1 = 0.0;
  return coef * (p1 - p0);
}

__device__ __forceinline__ double sixth_at(const double (*tile)[D6_W], int yl, double coef) {
  const double *c = &tile[threadIdx.y + D6_H][threadIdx.x + D6_H];
  double t = sixth_1d(c, 1, coef);
  if (yl > 1) t = t + sixth_1d(c, D6_W, coef);
  return t;
}

// Levels per block of k_diff6: the next level's four tiles are copied
// (cp.async, 8-byte) while the current level is filtered.
constexpr int D6_KC = 4;
constexpr int D6_NS = (D6_R * D6_W + D6_TX * D6_TY - 1) / (D6_TX * D6_TY);

// Index space (nx+1) x (ny+1) x ceil((nz+1) / D6_KC) in D6_TX x D6_TY blocks:
// the u, v, w and theta cells at (k, j, i) for the block's D6_KC levels.  The
// four fields' tiles (3-cell wrapped halo) of a level are staged together,
// double-buffered across levels, then filtered from shared memory.
// 5 resident blocks of 256 per SM (48 registers): 433 x 433 x 50, 0.886 vs
// 0.930 ms/step at the compiler's 62 registers (6: 1.089).
#ifndef WG_D6_MINB
#define WG_D6_MINB 5
#endif
#if WG_D6_MINB > 0
#define WG_D6_BOUNDS __launch_bounds__(D6_TX * D6_TY, WG_D6_MINB)
#else
#define WG_D6_BOUNDS __launch_bounds__(D6_TX * D6_TY)
#endif
__global__ void WG_D6_BOUNDS k_diff6(Grid g, Diff6Args a) {
  __shared__ double tile[2][4][D6_R][D6_W];
  const int i0 = blockIdx.x * D6_TX, j0 = blockIdx.y * D6_TY;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int k0 = blockIdx.z * D6_KC, k1 = min(nz + 1, k0 + D6_KC);
  const int tid = threadIdx.y * D6_TX + threadIdx.x;
  // this thread's tile elements and their wrapped in-plane offsets (mass / w,
  // u and v planes), resolved once for all levels
  int om[D6_NS], ou[D6_NS], ov[D6_NS];
#pragma unroll
  for (int n = 0; n < D6_NS; ++n) {
    const int e = tid + n * D6_TX * D6_TY;
    om[n] = ou[n] = ov[n] = -1;
    if (e < D6_R * D6_W) {
      const int r = e / D6_W, q = e - r * D6_W;
      const int jm = wrap(j0 - D6_H + r, ny), jv = wrap(j0 - D6_H + r, ny + 1);
      const int im = wrap(i0 - D6_H + q, nx), iu = wrap(i0 - D6_H + q, nx + 1);
      om[n] = jm * nx + im;
      ou[n] = jm * (nx + 1) + iu;
      ov[n] = jv * nx + im;
    }
  }
  auto issue = [&](int k, int b) {
    const bool mass_level = k < nz;
    const size_t pu = (size_t)k * (nx + 1) * ny, pv = (size_t)k * nx * (ny + 1), pm = (size_t)k * nx * ny;
    double *t = &tile[b][0][0][0];
    constexpr int TN = D6_R * D6_W;
#pragma unroll
    for (int n = 0; n < D6_NS; ++n) {
      if (om[n] < 0) continue;
      const int e = tid + n * D6_TX * D6_TY;
      cp_async8(t + 2 * TN + e, a.w + pm + om[n]);
      if (mass_level) {
        cp_async8(t + e, a.u + pu + ou[n]);
        cp_async8(t + TN + e, a.v + pv + ov[n]);
        cp_async8(t + 3 * TN + e, a.theta + pm + om[n]);
      }
    }
    cp_async_commit();
  };
  auto mu = [&](int jj, int ii) { return ld(a.mu, (size_t)jj * nx + ii); };
  issue(k0, 0);
  for (int k = k0; k < k1; ++k) {
    const int b = (k - k0) & 1;
    if (k + 1 < k1) {
      issue(k + 1, b ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const bool mass_level = k < nz;  // u, v, theta live on nz levels, w on nz + 1 (uniform over the block)
    const size_t pu = (size_t)k * (nx + 1) * ny, pv = (size_t)k * nx * (ny + 1), pm = (size_t)k * nx * ny;
    if (mass_level && i <= nx && j < ny) {  // u faces: mass_u from the edge-padded x average of mu
      const double muu = i == 0 ? mu(j, 0) : (i == nx ? mu(j, nx - 1) : 0.5 * (mu(j, i - 1) + mu(j, i)));
      const size_t c = pu + (size_t)j * (nx + 1) + i;
      a.u_tend[c] = a.u_tend[c] + (ld(g.c1h, k) * muu + ld(g.c2h, k)) * sixth_at(tile[b][0], ny, a.coef);
    }
    if (mass_level && i < nx && j <= ny) {  // v faces
      const double muv = j == 0 ? mu(0, i) : (j == ny ? mu(ny - 1, i) : 0.5 * (mu(j - 1, i) + mu(j, i)));
      const size_t c = pv + (size_t)j * nx + i;
      a.v_tend[c] = a.v_tend[c] + (ld(g.c1h, k) * muv + ld(g.c2h, k)) * sixth_at(tile[b][1], ny + 1, a.coef);
    }
    if (i < nx && j < ny) {
      const double mt = mu(j, i);
      const size_t c = pm + (size_t)j * nx + i;
      a.w_tend[c] = a.w_tend[c] + (ld(g.c1f, k) * mt + ld(g.c2f, k)) * sixth_at(tile[b][2], ny, a.coef);
      if (mass_level)
        a.t_tend[c] = a.t_tend[c] + (ld(g.c1h, k) * mt + ld(g.c2h, k)) * sixth_at(tile[b][3], ny, a.coef);
    }
    __syncthreads();  // buffer b is refilled two levels on
  }
}

}  // namespace wg
