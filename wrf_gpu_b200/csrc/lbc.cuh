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

template <typename FLD>
__device__ __forceinline__ double bounded(const LbcJob &a, const BdyLeaf &lf, FLD F, int k, int j, int i) {
  return a.ring ? lbc_value(a, lf, F, k, j, i) : F(j, i);
}

// Index space xl x yl x zl, blocks of LBC_THREADS threads.
constexpr int LBC_THREADS = 128;
__global__ void __launch_bounds__(LBC_THREADS) k_lbc_field(LbcJob a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const bool in = i < a.xl && j < a.yl;
  const size_t plane = (size_t)a.yl * a.xl;
  const size_t c = k * plane + (size_t)j * a.xl + i;
  const auto at = [&](int jj, int ii) { return k * plane + (size_t)jj * a.xl + ii; };
  if (a.x2 == nullptr) {
    if (a.pre == GUARD_THETA) {
      const GuardScalars gs = *a.gs;
      auto F = [&](int jj, int ii) { return guard_theta(ld(a.x, at(jj, ii)), ld(a.org, at(jj, ii)), gs); };
      double own = 0.0;
      if (in) {
        own = F(j, i) * guard_mass(ld(a.mu_next, (size_t)j * a.xl + i));
        double v = bounded(a, a.leaf, F, k, j, i);
        if (a.post == GUARD_FINITE && !isfinite(v)) v = ld(a.org, c);
        a.out[c] = v;
      }
      __shared__ double sh[LBC_THREADS / 32];
      const int tid = threadIdx.y * blockDim.x + threadIdx.x;
      // block_sum indexes warps by threadIdx.x: give it the flat thread index
      double s = own;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if ((tid & 31) == 0) sh[tid >> 5] = s;
      __syncthreads();
      if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < LBC_THREADS / 32; ++w) t += sh[w];
        a.after[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
      }
      return;
    }
    if (!in) return;
    double v;
    if (a.pre == GUARD_RATIO) {
      auto F = [&](int jj, int ii) {
        const double q = ld(a.x, at(jj, ii));
        return valid_ratio(q) ? q : ld(a.org, at(jj, ii));
      };
      v = bounded(a, a.leaf, F, k, j, i);
    } else {
      auto F = [&](int jj, int ii) { return ld(a.x, at(jj, ii)); };
      v = bounded(a, a.leaf, F, k, j, i);
    }
    if (a.clamp && v < 0.0) v = 0.0;  // jnp.maximum(v, 0): NaN stays NaN
    if (a.post == GUARD_FINITE && !isfinite(v)) v = ld(a.org, c);
    if (a.post == GUARD_RATIO && !valid_ratio(v)) v = ld(a.org, c);
    a.out[c] = v;
    return;
  }
  if (!in) return;
  double pert, base;
  if (a.pre == GUARD_MASS) {  // the dry-mass guard: total and perturbation from one source
    auto ok = [&](int jj, int ii) { return valid_mu(ld(a.x, at(jj, ii)), ld(a.x2, at(jj, ii))); };
    auto P = [&](int jj, int ii) { return ok(jj, ii) ? ld(a.x2, at(jj, ii)) : ld(a.org2, at(jj, ii)); };
    auto B = [&](int jj, int ii) {
      const size_t cc = at(jj, ii);
      return ok(jj, ii) ? ld(a.x, cc) - ld(a.x2, cc) : ld(a.org, cc) - ld(a.org2, cc);
    };
    pert = bounded(a, a.leaf, P, k, j, i);
    base = bounded(a, a.leaf2, B, k, j, i);
  } else {
    auto P = [&](int jj, int ii) { return ld(a.x2, at(jj, ii)); };
    auto B = [&](int jj, int ii) {
      const size_t cc = at(jj, ii);
      return ld(a.x, cc) - ld(a.x2, cc);
    };
    pert = bounded(a, a.leaf, P, k, j, i);
    base = bounded(a, a.leaf2, B, k, j, i);
  }
  // the boundary pass rebuilds every total as base + perturbation; without it
  // the (guarded) total is kept as it is
  double tot = base + pert;
  if (!a.ring) {
    const bool keep = a.pre != GUARD_MASS || valid_mu(ld(a.x, c), ld(a.x2, c));
    tot = keep ? ld(a.x, c) : ld(a.org, c);
  }
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

}  // namespace wg
