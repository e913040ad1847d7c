// Nest coupling around the step: the parent -> child boundary package and
// the child -> parent feedback (nesting/interp.py, nesting/
// boundary_construction.py, coupling/boundary_feedback.py).
//
//  * k_nest_interp: a parent field bilinearly gathered onto a child grid
//    with static per-row / per-column corner indices and weights, rows first
//    then columns (interp.py:248-277): f_y = (1 - wy) f[y0] + wy f[y1] at
//    the two corner columns, then (1 - wx) f_y[x0] + wx f_y[x1].
//  * k_nest_ring_leaf: one two-time boundary leaf (2, 4, width, z, side) of
//    the child (build_child_boundary_package, boundary_construction.py:
//    360-451): time 0 the child's own ring, time 1 the parent interpolated to
//    the same ring cells (or the child's own ring again for the base
//    leaves); W / E columns and S / N rows outer to inner, zero beyond the
//    field's extent or the leaf's (field_sides_3d, _fit).
//  * k_nest_feedback: the WRF copy_fcn overlap mean of each parent point's
//    child donors (boundary_feedback.py:362-425), written over a copy of the
//    parent; the sm121 1-2-1 smoother of the overlap interior as a j pass
//    into a scratch copy and an i pass back (:428-494); totals rebuilt as
//    parent base + fed-back perturbation (:557-568).
#pragma once
#include "dycore_common.cuh"

namespace wg {

struct NestInterp {
  const int *y0, *y1, *x0, *x1;
  const double *wy, *wx;
  int cny, cnx;  // child extent of this staggering
  int pny, pnx;  // parent extent of this staggering
};

__device__ __forceinline__ double nest_gather(const NestInterp &w, const double *parent, int z, int jj, int ii) {
  const size_t plane = (size_t)w.pny * w.pnx;
  const double *pz = parent + (size_t)z * plane;
  const int y0 = w.y0[jj], y1 = w.y1[jj], x0 = w.x0[ii], x1 = w.x1[ii];
  const double wy = w.wy[jj], wx = w.wx[ii];
  auto P = [&](int y, int x) { return __ldg(pz + (size_t)y * w.pnx + x); };
  const double fy0 = (1.0 - wy) * P(y0, x0) + wy * P(y1, x0);
  const double fy1 = (1.0 - wy) * P(y0, x1) + wy * P(y1, x1);
  return (1.0 - wx) * fy0 + wx * fy1;
}

// Index space (cnx, cny, nz): the full child grid.
__global__ void k_nest_interp(NestInterp w, const double *parent, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (i >= w.cnx || j >= w.cny) return;
  out[((size_t)z * w.cny + j) * w.cnx + i] = nest_gather(w, parent, z, j, i);
}

struct NestRingJob {
  NestInterp w;           // the gather of time 1 (ignored when !interp)
  int interp;             // 1: time 1 from the parent; 0: time 1 = time 0
  const double *parent;
  const double *child;    // (nzf, cny, cnx)
  const double *child_sub;  // nullable: the ring of child - child_sub (a base = total - perturbation)
  int nzf;                // levels of the field
  int width, side_len;    // strip geometry (field_sides_3d)
  int lz, lside;          // leaf extents (the fit)
  double *leaf;           // (2, 4, width, lz, lside)
};

// Index space (lside, width * 4, 2 * lz): every element of the leaf.
__global__ void k_nest_ring_leaf(NestRingJob a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int sb = blockIdx.y;             // side * width + b
  const int tz = blockIdx.z;             // t * lz + z
  if (q >= a.lside) return;
  const int side = sb / a.width, b = sb - side * a.width;
  const int t = tz / a.lz, z = tz - t * a.lz;
  const int cny = a.w.cny, cnx = a.w.cnx;
  const int xw = a.width < cnx ? a.width : cnx, yw = a.width < cny ? a.width : cny;
  double v = 0.0;
  int jj = -1, ii = -1;
  if (z < a.nzf && q < a.side_len) {
    if (side < 2 && b < xw && q < cny) {
      jj = q;
      ii = side == 0 ? b : cnx - 1 - b;
    } else if (side >= 2 && b < yw && q < cnx) {
      ii = q;
      jj = side == 2 ? b : cny - 1 - b;
    }
  }
  if (jj >= 0) {
    const size_t e = ((size_t)z * cny + jj) * cnx + ii;
    if (t == 1 && a.interp)
      v = nest_gather(a.w, a.parent, z, jj, ii);
    else
      v = a.child_sub != nullptr ? __ldg(a.child + e) - __ldg(a.child_sub + e) : __ldg(a.child + e);
  }
  a.leaf[((((size_t)t * 4 + side) * a.width + b) * a.lz + z) * a.lside + q] = v;
}

struct NestFeedback {
  const int *parent_lin, *child_lin;
  int npts, stencil, pwe, psn, cwe, csn;
};

// Index space (npts, nz): out (a copy of the parent) at the overlap points.
__global__ void k_nest_feedback(NestFeedback p, const double *child, double *out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y;
  if (n >= p.npts) return;
  const double *cz = child + (size_t)z * p.csn * p.cwe;
  const int *d = p.child_lin + (size_t)n * p.stencil;
  double acc = __ldg(cz + d[0]);
  for (int s = 1; s < p.stencil; ++s) acc = acc + __ldg(cz + d[s]);
  out[(size_t)z * p.psn * p.pwe + p.parent_lin[n]] = acc / (double)p.stencil;
}

// sm121 j pass: cnew (a copy of a) at the interior [j_lo, j_hi) x [i_lo, i_hi).
__global__ void k_sm121_j(const double *a, double *cnew, int ny, int nx, int i_lo, int i_hi, int j_lo, int j_hi) {
  const int i = i_lo + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = j_lo + blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (i >= i_hi || j >= j_hi) return;
  const double *az = a + (size_t)z * ny * nx;
  auto A = [&](int jj) { return az[(size_t)jj * nx + i]; };
  cnew[(size_t)z * ny * nx + (size_t)j * nx + i] = 0.25 * (A(j + 1) + 2.0 * A(j) + A(j - 1));
}

// sm121 i pass: out at the interior from cnew.
__global__ void k_sm121_i(const double *cnew, double *out, int ny, int nx, int i_lo, int i_hi, int j_lo, int j_hi) {
  const int i = i_lo + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = j_lo + blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (i >= i_hi || j >= j_hi) return;
  const double *cz = cnew + (size_t)z * ny * nx + (size_t)j * nx;
  out[(size_t)z * ny * nx + (size_t)j * nx + i] = 0.25 * (cz[i + 1] + 2.0 * cz[i] + cz[i - 1]);
}

// total = (parent total - parent perturbation) + new perturbation.
__global__ void k_nest_total(const double *ptot, const double *ppert, const double *npert, size_t n, double *out) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  out[e] = (__ldg(ptot + e) - __ldg(ppert + e)) + __ldg(npert + e);
}

}  // namespace wg
