// The end-of-step lateral boundary pass (apply_lateral_boundaries,
// coupling/boundary_apply.py:170-326): every forced field is relaxed in rows
// / columns 1..3 toward its boundary strips (WRF relax_bdytend as a value
// update, :589-663, each row computed from the unmodified field) and set to
// the strips in row / column 0 (:556-570; the S / N rows own the corners).
// One thread per cell of the field; a cell off the ring is copied.  A pair
// job relaxes a perturbation and its base (total - perturbation) and writes
// total = base + perturbation.  The post-step guards (guards.cuh) are fused
// on either side: `pre` guards the field as it is read (every neighbour the
// stencil reads sees the guarded value), `post` guards the value written.
#pragma once
#include "dycore_common.cuh"
#include "guards.cuh"

namespace wg {

enum { GUARD_NONE = 0, GUARD_THETA = 1, GUARD_RATIO = 2, GUARD_MASS = 3, GUARD_FINITE = 4 };

struct LbcJob {
  const double *x;   // the field (a pair: its total)
  const double *x2;  // a pair's perturbation, else null
  double *out;       // the new field (a pair: its total)
  double *out2;      // a pair's new perturbation
  BdyLeaf leaf;      // the field's strips (a pair: the perturbation's)
  BdyLeaf leaf2;     // a pair's base strips
  int zl, yl, xl;
  int ring;          // 0: no boundary pass, 1: ring 0 only (the specified cadence's pass), 2: ring 0 + relax rows
  int clamp;         // clip the bounded value at zero (moisture)
  double wf[4], wg[4];  // dt*fcx, dt*gcx of rows 1..3
  int all_ring;      // grids under 8 x 8: the ring kernel covers every cell, the elementwise one none
  int pre, post;     // GUARD_* before / after the boundary pass
  const double *org, *org2;  // the origin state's field (a pair: total, perturbation)
  const double *mu_next;     // the step output's mu_total (GUARD_THETA's mass weight)
  const GuardScalars *gs;    // the limiter's domain scalars (GUARD_THETA)
  double *after;             // per-block partials of the limited theta * mass (GUARD_THETA)
};

// The new value of one field at (k, j, i) on the ring; F(jj, ii) reads the field.
template <typename FLD>
__device__ __forceinline__ double lbc_value(const LbcJob &a, const BdyLeaf &lf, FLD F, int k, int j, int i) {
  const int zl = a.zl, yl = a.yl, xl = a.xl;
  // spec ring, written W, E, S, N: the last writer wins (the rows own the corners)
  if (j == yl - 1) return strip_at(lf, zl, 3, 0, k, i);
  if (j == 0) return strip_at(lf, zl, 2, 0, k, i);
  if (i == xl - 1) return strip_at(lf, zl, 1, 0, k, j);
  if (i == 0) return strip_at(lf, zl, 0, 0, k, j);
  if (a.ring < 2) return F(j, i);
  // the relax-zone owner (sides written W, E, S, N; the last writer wins): S / N
  // rows b own columns [b, xl-1-b], W / E columns b own rows [b+1, yl-2-b]
  int side = -1, b = 0;
  const int bs = j, bn = yl - 1 - j, bw = i, be = xl - 1 - i;
  if (bn >= 1 && bn <= 3 && i >= bn && i <= xl - 1 - bn) { side = 3; b = bn; }
  else if (bs >= 1 && bs <= 3 && i >= bs && i <= xl - 1 - bs) { side = 2; b = bs; }
  else if (be >= 1 && be <= 3 && j >= be + 1 && j <= yl - 2 - be) { side = 1; b = be; }
  else if (bw >= 1 && bw <= 3 && j >= bw + 1 && j <= yl - 2 - bw) { side = 0; b = bw; }
  if (side < 0) return F(j, i);
  double cur, te, ti, f1, f2, s0, se, si;
  if (side >= 2) {  // tangential x
    const int je = (side == 2) ? j - 1 : j + 1, jin = (side == 2) ? j + 1 : j - 1;
    const int il = i > 0 ? i - 1 : 0, ir = i < xl - 1 ? i + 1 : xl - 1;
    cur = F(j, i);
    te = F(je, i);
    ti = F(jin, i);
    s0 = strip_at(lf, zl, side, b, k, i);
    f1 = strip_at(lf, zl, side, b, k, il) - F(j, il);
    f2 = strip_at(lf, zl, side, b, k, ir) - F(j, ir);
    se = strip_at(lf, zl, side, b - 1, k, i);
    si = strip_at(lf, zl, side, b + 1, k, i);
  } else {  // tangential y
    const int ie = (side == 0) ? i - 1 : i + 1, iin = (side == 0) ? i + 1 : i - 1;
    const int jl = j > 0 ? j - 1 : 0, jr = j < yl - 1 ? j + 1 : yl - 1;
    cur = F(j, i);
    te = F(j, ie);
    ti = F(j, iin);
    s0 = strip_at(lf, zl, side, b, k, j);
    f1 = strip_at(lf, zl, side, b, k, jl) - F(jl, i);
    f2 = strip_at(lf, zl, side, b, k, jr) - F(jr, i);
    se = strip_at(lf, zl, side, b - 1, k, j);
    si = strip_at(lf, zl, side, b + 1, k, j);
  }
  const double fls0 = s0 - cur;
  const double fls3 = se - te, fls4 = si - ti;
  // the reference's fls1 / fls2 are fls0 shifted by -1 / +1 along the row (clamped)
  const double lap = f1 + f2 + fls3 + fls4 - 4.0 * fls0;
  return cur + a.wf[b] * fls0 - a.wg[b] * lap;
}

constexpr int LBC_THREADS = 128;
constexpr int LBC_RING_THREADS = 128;
constexpr int LBC_THREADS_MAX = 128;
constexpr int LBC_KZ = 4;

// The post guards of a written pair (total, perturbation), then the stores.
__device__ __forceinline__ void post_pair(const LbcJob &a, double tot, double pert, size_t c) {
  if (a.post == GUARD_FINITE) {
    if (!isfinite(tot)) tot = ld(a.org, c);
    if (!isfinite(pert)) pert = ld(a.org2, c);
  } else if (a.post == GUARD_MASS && !valid_mu(tot, pert)) {
    tot = ld(a.org, c);
    pert = ld(a.org2, c);
  }
  a.out[c] = tot;
  a.out2[c] = pert;
}

// The post guard of one written value.
__device__ __forceinline__ double post_single(const LbcJob &a, double v, size_t c) {
  if (a.post == GUARD_FINITE && !isfinite(v)) v = ld(a.org, c);
  if (a.post == GUARD_RATIO && !valid_ratio(v)) v = ld(a.org, c);
  return v;
}

// The per-block partial of sum(limited theta * mass) (GUARD_THETA jobs);
// `own` is this thread's sum of the limited theta over its levels, `m` its
// column's mass weight.
__device__ __forceinline__ void theta_partial(const LbcJob &a, double own, double m, size_t slot) {
  __shared__ double sh[LBC_THREADS_MAX / 32];
  double s = own * m;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nt = blockDim.x * blockDim.y;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((tid & 31) == 0) sh[tid >> 5] = s;
  __syncthreads();
  if (tid == 0) {
    double tsum = 0.0;
    for (int w = 0; w < nt / 32; ++w) tsum += sh[w];
    a.after[slot] = tsum;
  }
}

// The elementwise part: index space xl x yl, each thread one column in
// chunks of LBC_KZ levels with each chunk's loads issued first.  With the
// boundary pass the 4-wide ring band is left to lbc_ring.
__device__ __forceinline__ void lbc_field(const LbcJob &a, int bx, int by, size_t slot) {
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int xl = a.xl, yl = a.yl, zl = a.zl;
  const bool in = i < xl && j < yl && (!a.ring || (i >= 4 && i < xl - 4 && j >= 4 && j < yl - 4));
  const size_t plane = (size_t)yl * xl;
  const bool th = a.pre == GUARD_THETA;
  double own = 0.0;
  if (in && a.x2 == nullptr) {
    const double *x = a.x + (size_t)j * xl + i;
    const double *org = a.org + (size_t)j * xl + i;
    double *out = a.out + (size_t)j * xl + i;
    GuardScalars gs{};
    if (th) gs = *a.gs;
    for (int k0 = 0; k0 < zl; k0 += LBC_KZ) {
      const int nk = zl - k0 < LBC_KZ ? zl - k0 : LBC_KZ;
      double xv[LBC_KZ], ov[LBC_KZ];
#pragma unroll
      for (int t = 0; t < LBC_KZ; ++t)
        if (t < nk) {
          xv[t] = ld(x, (size_t)(k0 + t) * plane);
          ov[t] = th ? ld(org, (size_t)(k0 + t) * plane) : 0.0;
        }
#pragma unroll
      for (int t = 0; t < LBC_KZ; ++t) {
        if (t >= nk) break;
        const size_t c = (size_t)(k0 + t) * plane;
        double v = xv[t];
        if (th) v = guard_theta(v, ov[t], gs);
        else if (a.pre == GUARD_RATIO && !valid_ratio(v)) v = ld(org, c);
        own += v;
        if (a.clamp && v < 0.0) v = 0.0;  // jnp.maximum(v, 0): NaN stays NaN
        if (a.post == GUARD_FINITE && !isfinite(v)) v = ld(org, c);
        if (a.post == GUARD_RATIO && !valid_ratio(v)) v = ld(org, c);
        out[c] = v;
      }
    }
  } else if (in) {
    // a pair: the boundary pass rebuilds every total as base + perturbation;
    // without it the (guarded) total is kept as it is
    const size_t c0 = (size_t)j * xl + i;
    for (int k0 = 0; k0 < zl; k0 += LBC_KZ) {
      const int nk = zl - k0 < LBC_KZ ? zl - k0 : LBC_KZ;
      double tv[LBC_KZ], pv[LBC_KZ];
#pragma unroll
      for (int t = 0; t < LBC_KZ; ++t)
        if (t < nk) {
          tv[t] = ld(a.x, c0 + (size_t)(k0 + t) * plane);
          pv[t] = ld(a.x2, c0 + (size_t)(k0 + t) * plane);
        }
#pragma unroll
      for (int t = 0; t < LBC_KZ; ++t) {
        if (t >= nk) break;
        const size_t c = c0 + (size_t)(k0 + t) * plane;
        double tot = tv[t], pert = pv[t];
        if (a.pre == GUARD_MASS && !valid_mu(tot, pert)) {
          tot = ld(a.org, c);
          pert = ld(a.org2, c);
        }
        if (a.ring) tot = (tot - pert) + pert;
        post_pair(a, tot, pert, c);
      }
    }
  }
  if (th) theta_partial(a, own, in ? guard_mass(ld(a.mu_next, (size_t)j * xl + i)) : 0.0, slot);
}

// Cells of the 4-wide ring band per level: rows 0..3 and yl-4..yl-1 (all
// columns), then columns 0..3 and xl-4..xl-1 of rows 4..yl-5, row by row
// (xl, yl >= 8); every cell when all_ring.
__host__ __device__ inline int ring_cells(int xl, int yl, int all_ring) {
  return all_ring ? xl * yl : 8 * xl + 8 * (yl - 8);
}

// The stencil part: index space ring_cells x zl, one thread per band cell.
__device__ __forceinline__ void lbc_ring(const LbcJob &a, int bx, int k, size_t slot) {
  const int xl = a.xl, yl = a.yl;
  const int r = bx * blockDim.x + threadIdx.x;
  const int nb = ring_cells(xl, yl, a.all_ring);
  int i = 0, j = 0;
  const bool in = r < nb;
  if (in) {
    if (a.all_ring) {
      j = r / xl;
      i = r - j * xl;
    } else if (r < 8 * xl) {
      const int row = r / xl;
      i = r - row * xl;
      j = row < 4 ? row : yl - 8 + row;
    } else {  // eight band columns of one row per 8 threads (two 32-byte runs)
      const int q = r - 8 * xl;
      const int col = q & 7;
      j = 4 + (q >> 3);
      i = col < 4 ? col : xl - 8 + col;
    }
  }
  const size_t plane = (size_t)yl * xl;
  const auto at = [&](int jj, int ii) { return (size_t)k * plane + (size_t)jj * xl + ii; };
  const bool th = a.pre == GUARD_THETA;
  double own = 0.0;
  if (in && a.x2 == nullptr) {
    GuardScalars gs{};
    if (th) gs = *a.gs;
    auto F = [&](int jj, int ii) {
      const size_t cc = at(jj, ii);
      const double x = ld(a.x, cc);
      if (th) return guard_theta(x, ld(a.org, cc), gs);
      if (a.pre == GUARD_RATIO && !valid_ratio(x)) return ld(a.org, cc);
      return x;
    };
    own = F(j, i);
    double v = lbc_value(a, a.leaf, F, k, j, i);
    if (a.clamp && v < 0.0) v = 0.0;
    a.out[at(j, i)] = post_single(a, v, at(j, i));
  } else if (in) {
    auto ok = [&](int jj, int ii) {
      return a.pre != GUARD_MASS || valid_mu(ld(a.x, at(jj, ii)), ld(a.x2, at(jj, ii)));
    };
    auto P = [&](int jj, int ii) { return ok(jj, ii) ? ld(a.x2, at(jj, ii)) : ld(a.org2, at(jj, ii)); };
    auto B = [&](int jj, int ii) {
      const size_t cc = at(jj, ii);
      return ok(jj, ii) ? ld(a.x, cc) - ld(a.x2, cc) : ld(a.org, cc) - ld(a.org2, cc);
    };
    double pert = lbc_value(a, a.leaf, P, k, j, i);
    double tot = lbc_value(a, a.leaf2, B, k, j, i) + pert;
    post_pair(a, tot, pert, at(j, i));
  }
  if (th) theta_partial(a, own, in ? guard_mass(ld(a.mu_next, (size_t)j * xl + i)) : 0.0, slot);
}

// Every field of one epilogue in one launch.  All jobs share the x / y grid
// (sized for the widest field; threads past a field's extent idle);
// blockIdx.z is the job of the elementwise kernel, and the ring kernel's
// blockIdx.y is flattened over the jobs' levels: job q owns [start[q], start[q+1]).  The theta
// job's partial of a block goes to slot slot0[q] + its index within the job.
constexpr int LBC_MAX_JOBS = 16;
struct LbcBatch {
  LbcJob job[LBC_MAX_JOBS];
  int start[LBC_MAX_JOBS + 1];
  int slot0[LBC_MAX_JOBS];
  int njobs;
};

__device__ __forceinline__ int batch_job(const LbcBatch &b, int blk) {
  int q = 0;
  while (q + 1 < b.njobs && blk >= b.start[q + 1]) ++q;
  return q;
}

__global__ void __launch_bounds__(LBC_THREADS, 8) k_lbc_fields(const __grid_constant__ LbcBatch b) {
  const int q = blockIdx.z;
  lbc_field(b.job[q], blockIdx.x, blockIdx.y, (size_t)b.slot0[q] + (size_t)blockIdx.y * gridDim.x + blockIdx.x);
}

__global__ void __launch_bounds__(LBC_RING_THREADS) k_lbc_rings(const __grid_constant__ LbcBatch b) {
  const int q = batch_job(b, blockIdx.y);
  const int k = blockIdx.y - b.start[q];
  lbc_ring(b.job[q], blockIdx.x, k, (size_t)b.slot0[q] + (size_t)k * gridDim.x + blockIdx.x);
}

}  // namespace wg
