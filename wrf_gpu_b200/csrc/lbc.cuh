// The end-of-step lateral boundary pass (apply_lateral_boundaries,
// coupling/boundary_apply.py:170-326): every forced field is relaxed in rows
// / columns 1..3 toward its boundary strips (WRF relax_bdytend as a value
// update, :589-663, each row computed from the unmodified field) and set to
// the strips in row / column 0 (:556-570; the S / N rows own the corners).
// One thread per cell of the field; a cell off the ring is copied.  A pair
// job relaxes a perturbation and its base (total - perturbation) and writes
// total = base + perturbation.
#pragma once
#include "dycore_common.cuh"

namespace wg {

struct LbcJob {
  const double *x;   // the field (a pair: its total)
  const double *x2;  // a pair's perturbation, else null
  double *out;       // the new field (a pair: its total)
  double *out2;      // a pair's new perturbation
  BdyLeaf leaf;      // the field's strips (a pair: the perturbation's)
  BdyLeaf leaf2;     // a pair's base strips
  int zl, yl, xl;
  int relax;         // 0: ring 0 only (the specified cadence's end-of-step pass)
  int clamp;         // clip the result at zero (moisture)
  double wf[4], wg[4];  // dt*fcx, dt*gcx of rows 1..3
};

// The new value of one field at (k, j, i); F(jj, ii) reads the unmodified field.
template <typename FLD>
__device__ __forceinline__ double lbc_value(const LbcJob &a, const BdyLeaf &lf, FLD F, int k, int j, int i) {
  const int zl = a.zl, yl = a.yl, xl = a.xl;
  // spec ring, written W, E, S, N: the last writer wins (the rows own the corners)
  if (j == yl - 1) return strip_at(lf, zl, 3, 0, k, i);
  if (j == 0) return strip_at(lf, zl, 2, 0, k, i);
  if (i == xl - 1) return strip_at(lf, zl, 1, 0, k, j);
  if (i == 0) return strip_at(lf, zl, 0, 0, k, j);
  if (!a.relax) return F(j, i);
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

// Index space xl x yl x zl.
__global__ void k_lbc_field(LbcJob a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= a.xl || j >= a.yl) return;
  const size_t plane = (size_t)a.yl * a.xl;
  const size_t c = k * plane + (size_t)j * a.xl + i;
  if (a.x2 == nullptr) {
    auto F = [&](int jj, int ii) { return ld(a.x, k * plane + (size_t)jj * a.xl + ii); };
    double v = lbc_value(a, a.leaf, F, k, j, i);
    if (a.clamp) v = dmax(v, 0.0);
    a.out[c] = v;
    return;
  }
  auto P = [&](int jj, int ii) { return ld(a.x2, k * plane + (size_t)jj * a.xl + ii); };
  auto B = [&](int jj, int ii) {
    const size_t cc = k * plane + (size_t)jj * a.xl + ii;
    return ld(a.x, cc) - ld(a.x2, cc);
  };
  const double pert = lbc_value(a, a.leaf, P, k, j, i);
  const double base = lbc_value(a, a.leaf2, B, k, j, i);
  a.out[c] = base + pert;
  a.out2[c] = pert;
}

}  // namespace wg
