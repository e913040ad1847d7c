// The forecast step's post-step guards (runtime/operational_mode.py:
// 1300-1520, applied at :4950-4983):
//  * theta increment limiter (_positive_definite_theta_increment_limiter,
//    :1387-1455): cells whose theta is non-finite or outside [0, 1000] K get
//    the RK increment scaled back into the interval; the removed mass-weighted
//    increment is spread over every cell in proportion to its room, so the
//    domain integral of theta * mu_total is kept.  Three reductions: the
//    target and limited integrals and the room (k_guard_reduce, fixed grid,
//    per-block partials, one-block k_guard_finalize: deterministic order), then
//    the per-cell result (guard_theta, evaluated where the field is written)
//    and its integral (k_guard_diag over the writer's per-block partials);
//  * dry-mass guard (_limit_guarded_mass_state, :1458-1470): mu_total and mu'
//    fall back to the origin together where either is non-finite or
//    mu_total < 1 Pa;
//  * mixing-ratio guard (_valid_mixing_ratio, :1300-1306): outside
//    [0, 0.05] or non-finite falls back to the origin;
//  * finite guard (_finite_or_origin, :1309-1314).
#pragma once
#include <climits>

#include "../../include/wrfgpu.h"
#include "dycore_common.cuh"

namespace wg {

constexpr double THETA_LIM_MIN_K = 0.0;     // operational_mode.py:180
constexpr double THETA_LIM_MAX_K = 1000.0;  // operational_mode.py:198
constexpr double MIXING_RATIO_MAX = 0.05;   // operational_mode.py:1300
constexpr int GUARD_THREADS = 256;

// Per-block partials of k_guard_reduce.
struct GuardPartial {
  double target, mass0, cap_add, cap_sub;
  long long count, first;
};

// The limiter's domain scalars, written by k_guard_finalize.
struct GuardScalars {
  double target, mass0;
  double sf;  // sign(residual) * fraction
  int res_nonneg;
  long long count, first;
};

// One cell of the limiter before the redistribution: the finite candidate
// and the scaled-back value (lim0); *limited is set when the cell offends.
__device__ __forceinline__ void theta_lim0(double c, double o, double *fc, double *lim0, bool *limited) {
  const double lo = THETA_LIM_MIN_K, hi = THETA_LIM_MAX_K, mid = 0.5 * (lo + hi);
  double so = isfinite(o) ? o : mid;
  so = fmin(fmax(so, lo), hi);
  const bool fin = isfinite(c);
  const double f = fin ? c : so;
  const double raw = f - so;
  const bool lim = !fin || f > hi || f < lo;
  double alpha = 1.0;
  if (lim) {
    const double a = raw > 0.0 ? (hi - so) / raw : (raw < 0.0 ? (lo - so) / raw : 1.0);
    alpha = fmin(fmax(a, 0.0), 1.0);
  }
  *fc = f;
  *lim0 = so + alpha * raw;
  *limited = lim;
}

// The limited theta of one cell from the domain scalars.
__device__ __forceinline__ double guard_theta(double c, double o, const GuardScalars &s) {
  double fc, l0;
  bool lim;
  theta_lim0(c, o, &fc, &l0, &lim);
  const double room = s.res_nonneg ? THETA_LIM_MAX_K - l0 : l0 - THETA_LIM_MIN_K;
  const double v = l0 + s.sf * room;
  return fmin(fmax(v, THETA_LIM_MIN_K), THETA_LIM_MAX_K);
}

// The theta mass weight: the column's mu_total where finite and positive.
__device__ __forceinline__ double guard_mass(double mu) { return (isfinite(mu) && mu > 0.0) ? mu : 0.0; }

__device__ __forceinline__ bool valid_ratio(double q) { return isfinite(q) && q >= 0.0 && q <= MIXING_RATIO_MAX; }

__device__ __forceinline__ bool valid_mu(double total, double pert) {
  return isfinite(total) && isfinite(pert) && total >= 1.0;
}

// Deterministic block sum of one double (fixed shuffle tree, then warps in order).
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < NT / 32; ++w) t += sh[w];
  return t;  // valid in thread 0
}

template <int NT>
__device__ __forceinline__ long long block_sum_ll(long long v, long long *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  long long t = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < NT / 32; ++w) t += sh[w];
  return t;
}

template <int NT>
__device__ __forceinline__ long long block_min_ll(long long v, long long *sh) {
  for (int o = 16; o > 0; o >>= 1) {
    const long long u = __shfl_down_sync(0xffffffffu, v, o);
    v = u < v ? u : v;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  long long t = v;
  if (threadIdx.x == 0)
    for (int w = 0; w < NT / 32; ++w) t = sh[w] < t ? sh[w] : t;
  return t;
}

// Pass 1: per-block partials of the target integral sum(fc * m), the
// scaled-back integral sum(lim0 * m), both rooms, the offending count and the
// first offending flat index.  Grid-stride over the nz*ny*nx mass cells.
__global__ void __launch_bounds__(GUARD_THREADS) k_guard_reduce(const double *theta, const double *origin,
                                                                 const double *mu_total, int nz, int ny, int nx,
                                                                 GuardPartial *part) {
  __shared__ double shd[GUARD_THREADS / 32];
  __shared__ long long shl[GUARD_THREADS / 32];
  const long long n = (long long)nz * ny * nx, plane = (long long)ny * nx;
  double t = 0.0, m0 = 0.0, ca = 0.0, cs = 0.0;
  long long cnt = 0, first = LLONG_MAX;
  for (long long c = (long long)blockIdx.x * GUARD_THREADS + threadIdx.x; c < n;
       c += (long long)gridDim.x * GUARD_THREADS) {
    const double m = guard_mass(ld(mu_total, (size_t)(c % plane)));
    double fc, l0;
    bool lim;
    theta_lim0(ld(theta, (size_t)c), ld(origin, (size_t)c), &fc, &l0, &lim);
    t += fc * m;
    m0 += l0 * m;
    ca += (THETA_LIM_MAX_K - l0) * m;
    cs += (l0 - THETA_LIM_MIN_K) * m;
    if (lim) {
      ++cnt;
      first = c < first ? c : first;
    }
  }
  GuardPartial r;
  r.target = block_sum<GUARD_THREADS>(t, shd);
  r.mass0 = block_sum<GUARD_THREADS>(m0, shd);
  r.cap_add = block_sum<GUARD_THREADS>(ca, shd);
  r.cap_sub = block_sum<GUARD_THREADS>(cs, shd);
  r.count = block_sum_ll<GUARD_THREADS>(cnt, shl);
  r.first = block_min_ll<GUARD_THREADS>(first, shl);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

// Pass 2 (one block): the domain scalars from k_guard_reduce's partials.
__global__ void __launch_bounds__(GUARD_THREADS) k_guard_finalize(const GuardPartial *part, int nparts,
                                                                   GuardScalars *s) {
  __shared__ double shd[GUARD_THREADS / 32];
  __shared__ long long shl[GUARD_THREADS / 32];
  double t = 0.0, m0 = 0.0, ca = 0.0, cs = 0.0;
  long long cnt = 0, first = LLONG_MAX;
  for (int b = threadIdx.x; b < nparts; b += GUARD_THREADS) {
    const GuardPartial &p = part[b];
    t += p.target;
    m0 += p.mass0;
    ca += p.cap_add;
    cs += p.cap_sub;
    cnt += p.count;
    first = p.first < first ? p.first : first;
  }
  t = block_sum<GUARD_THREADS>(t, shd);
  m0 = block_sum<GUARD_THREADS>(m0, shd);
  ca = block_sum<GUARD_THREADS>(ca, shd);
  cs = block_sum<GUARD_THREADS>(cs, shd);
  cnt = block_sum_ll<GUARD_THREADS>(cnt, shl);
  first = block_min_ll<GUARD_THREADS>(first, shl);
  if (threadIdx.x == 0) {
    const double res = t - m0;
    const bool nonneg = res >= 0.0;
    const double cap = nonneg ? ca : cs;
    const double frac = cap > 0.0 ? fmin(fabs(res) / cap, 1.0) : 0.0;
    const double sgn = res > 0.0 ? 1.0 : (res < 0.0 ? -1.0 : 0.0);
    s->target = t;
    s->mass0 = m0;
    s->sf = sgn * frac;
    s->res_nonneg = nonneg ? 1 : 0;
    s->count = cnt;
    s->first = first;
  }
}

// Pass 3 (one block): the limited integral from the theta writer's per-block
// partials, and the diagnostics record.
__global__ void __launch_bounds__(GUARD_THREADS) k_guard_diag(const double *after_part, int nparts,
                                                               const GuardScalars *s, int ny, int nx,
                                                               wrfgpu_theta_limiter_diag *diag) {
  __shared__ double shd[GUARD_THREADS / 32];
  double a = 0.0;
  for (int b = threadIdx.x; b < nparts; b += GUARD_THREADS) a += after_part[b];
  a = block_sum<GUARD_THREADS>(a, shd);
  if (threadIdx.x == 0) {
    diag->limited_cell_count = (int)s->count;
    if (s->count > 0) {
      const long long plane = (long long)ny * nx, f = s->first;
      const long long z = f / plane, rem = f - z * plane, y = rem / nx;
      diag->first_limited_cell_xyz[0] = (int)(rem - y * nx);
      diag->first_limited_cell_xyz[1] = (int)y;
      diag->first_limited_cell_xyz[2] = (int)z;
    } else {
      diag->first_limited_cell_xyz[0] = diag->first_limited_cell_xyz[1] = diag->first_limited_cell_xyz[2] = -1;
    }
    diag->mass_before = s->target;
    diag->mass_after = a;
    diag->mass_residual = a - s->target;
  }
}

// The guards-off record (_empty_theta_limiter_diagnostics, :1374-1384).
__global__ void k_guard_diag_empty(wrfgpu_theta_limiter_diag *diag) {
  diag->limited_cell_count = 0;
  diag->first_limited_cell_xyz[0] = diag->first_limited_cell_xyz[1] = diag->first_limited_cell_xyz[2] = -1;
  diag->mass_before = diag->mass_after = diag->mass_residual = 0.0;
}

}  // namespace wg
