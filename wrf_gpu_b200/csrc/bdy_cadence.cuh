// The specified-domain boundary cadence (operational namelist
// specified_bdy_cadence; operational_mode.py:1984-2041, 2478-2530, 3085-3092;
// coupling/boundary_apply.py:948-1043, 1148-1340; core/acoustic.py:383-516,
// 777-785, 902-915, 1059-1090) and the nested child's in-loop forcings
// (force_geopotential off; operational_mode.py:1906-1968;
// boundary_apply.py:1045-1087).  Everything here touches only the outer five
// rows / columns of the domain, so the kernels run over ring cells only:
//   * k_spec_relax_add    -- WRF relax_bdy_dry: the relax-zone (rings 1..3)
//                            tendencies of the coupled u, v, theta, ph', mu'
//                            and w toward the boundary leaves, added to the
//                            stage tendencies.  The cadence relaxes u, v,
//                            theta, ph' and mu' (mu' into the first stage's
//                            tendency only) from the step-start state; the
//                            nested child ph' and / or w from the stage state
//                            with the stage mass;
//   * k_spec_w_zero_grad  -- WRF zero_grad_bdy for w, every acoustic substep:
//                            the ring-0 work w whose finished physical w equals
//                            the nearest interior physical w.
// The ring-0 pins of the tangential winds (advance_uv), of mu / muts / muave,
// the work theta and ph (the column kernel) use ring_target / strip_at inline.
#pragma once
#include "dycore_common.cuh"

namespace wg {

// Relax-zone rows of the default boundary configuration (spec_zone 1, relax_zone 4).
constexpr int RELAX_B0 = 1, RELAX_B1 = 4;

// Relaxed fields, in the order of RelaxArgs::fields.
enum RelaxField { RELAX_U = 0, RELAX_V, RELAX_THETA, RELAX_PH, RELAX_MU, RELAX_W, RELAX_NFIELD };

struct RelaxArgs {
  // the relax reference: fields and the total dry mass that couples them
  const double *u, *v, *theta, *ph_pert, *mu_total, *mu_pert, *w;
  BdyLeaf lu, lv, lt, lph, lmu, lw;  // leaves at the step's lead
  // per-second weights fcx, gcx of rows b = 1..3 (index b)
  double fcx[RELAX_B1], gcx[RELAX_B1];
  // tendencies the relax terms are added to (mu_tend: the first stage only, else null)
  double *u_tend, *v_tend, *t_tend, *ph_tend, *mu_tend, *rw_tend;
  // the relaxed fields of this launch (RelaxField values); blockIdx.z / (nz+1) indexes them
  int nfield;
  int fields[RELAX_NFIELD];
};

// Ring position e of row / column ring b of a (yl, xl) field in WRF's relax
// order: the S and N rows own the corners (i in [b, xl-1-b]), the W and E
// columns take rows [b+1, yl-2-b].  Returns false past the ring.  side: 0 W,
// 1 E, 2 S, 3 N.
__device__ __forceinline__ bool relax_ring_cell(int e, int b, int yl, int xl, int &j, int &i, int &side) {
  const int ns = xl - 2 * b, nw = yl - 2 - 2 * b;
  if (ns <= 0) return false;
  if (e < ns) { side = 2; j = b; i = b + e; return true; }
  e -= ns;
  if (e < ns) { side = 3; j = yl - 1 - b; i = b + e; return true; }
  e -= ns;
  if (nw <= 0) return false;
  if (e < nw) { side = 0; i = b; j = b + 1 + e; return true; }
  e -= nw;
  if (e < nw) { side = 1; i = xl - 1 - b; j = b + 1 + e; return true; }
  return false;
}

// One relax_bdytend value (boundary_apply.py:972-1006): FLS(jj, ii) is the
// coupled residual target - field; the tangential neighbours are clamped.
template <typename FLS>
__device__ __forceinline__ double relax_value(FLS fls, int side, int j, int i, int yl, int xl, double fcx,
                                              double gcx) {
  const double f0 = fls(j, i);
  double f1, f2, f3, f4;
  if (side >= 2) {  // S / N row: tangential x, normal y
    const int je = (side == 2) ? j - 1 : j + 1, jin = (side == 2) ? j + 1 : j - 1;
    f1 = fls(j, i > 0 ? i - 1 : 0);
    f2 = fls(j, i < xl - 1 ? i + 1 : xl - 1);
    f3 = fls(je, i);
    f4 = fls(jin, i);
  } else {  // W / E column: tangential y, normal x
    const int ie = (side == 0) ? i - 1 : i + 1, iin = (side == 0) ? i + 1 : i - 1;
    f1 = fls(j > 0 ? j - 1 : 0, i);
    f2 = fls(j < yl - 1 ? j + 1 : yl - 1, i);
    f3 = fls(j, ie);
    f4 = fls(j, iin);
  }
  const double lap = f1 + f2 + f3 + f4 - 4.0 * f0;
  return fcx * f0 - gcx * lap;
}

// blockIdx.y = ring b - 1, blockIdx.z = slot * (nz + 1) + level with
// fields[slot] the relaxed field; x threads over the ring positions.
__global__ void k_spec_relax_add(Grid g, RelaxArgs a) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int b = RELAX_B0 + blockIdx.y;
  const int slot = blockIdx.z / (nz + 1), k = blockIdx.z - slot * (nz + 1);
  if (slot >= a.nfield) return;
  const int field = a.fields[slot];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  int zl, yl, xl;
  switch (field) {
    case RELAX_U: zl = nz; yl = ny; xl = nx + 1; break;
    case RELAX_V: zl = nz; yl = ny + 1; xl = nx; break;
    case RELAX_THETA: zl = nz; yl = ny; xl = nx; break;
    case RELAX_PH: case RELAX_W: zl = nz + 1; yl = ny; xl = nx; break;
    default: zl = 1; yl = ny; xl = nx; break;
  }
  if (k >= zl || (field == RELAX_MU && a.mu_tend == nullptr)) return;
  int j, i, side;
  if (!relax_ring_cell(e, b, yl, xl, j, i, side)) return;
  auto mu = [&](int jj, int ii) { return ld(a.mu_total, ix2(jj, ii, nx)); };
  double val;
  if (field == RELAX_U) {
    const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
    auto fls = [&](int jj, int ii) {
      // face mass of the relax reference (edge-padded face average)
      const double muu = 0.5 * (mu(jj, ii > 0 ? ii - 1 : 0) + mu(jj, ii < nx ? ii : nx - 1));
      const double mass = c1 * muu + c2;
      const size_t f2 = ix2(jj, ii, nx + 1);
      const double tgt = div_msf(mass * ring_target(a.lu, zl, yl, xl, k, jj, ii), g.msfuy, g.rmsfuy, f2);
      const double fld = div_msf(mass * ld(a.u, ix3(k, jj, ii, ny, nx + 1)), g.msfuy, g.rmsfuy, f2);
      return tgt - fld;
    };
    val = 0.0 + relax_value(fls, side, j, i, yl, xl, a.fcx[b], a.gcx[b]);
    double *t = a.u_tend + ix3(k, j, i, ny, nx + 1);
    *t = *t + val;
  } else if (field == RELAX_V) {
    const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
    auto fls = [&](int jj, int ii) {
      const double muv = 0.5 * (mu(jj > 0 ? jj - 1 : 0, ii) + mu(jj < ny ? jj : ny - 1, ii));
      const double mass = c1 * muv + c2;
      const size_t f2 = ix2(jj, ii, nx);
      const double tgt = div_msf(mass * ring_target(a.lv, zl, yl, xl, k, jj, ii), g.msfvx, g.rmsfvx, f2);
      const double fld = div_msf(mass * ld(a.v, ix3(k, jj, ii, ny + 1, nx)), g.msfvx, g.rmsfvx, f2);
      return tgt - fld;
    };
    val = 0.0 + relax_value(fls, side, j, i, yl, xl, a.fcx[b], a.gcx[b]);
    double *t = a.v_tend + ix3(k, j, i, ny + 1, nx);
    *t = *t + val;
  } else if (field == RELAX_THETA) {
    const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
    auto fls = [&](int jj, int ii) {
      const double mass = c1 * mu(jj, ii) + c2;
      return mass * ring_target(a.lt, zl, yl, xl, k, jj, ii) - mass * ld(a.theta, ix3(k, jj, ii, ny, nx));
    };
    val = div_msf(0.0 + relax_value(fls, side, j, i, yl, xl, a.fcx[b], a.gcx[b]), g.msfty, g.rmsfty, ix2(j, i, nx));
    double *t = a.t_tend + ix3(k, j, i, ny, nx);
    *t = *t + val;
  } else if (field == RELAX_PH || field == RELAX_W) {
    // full-level fields coupled with c1f*mu+c2f (boundary_apply.py:1062-1068, 1081-1087)
    const bool ph = field == RELAX_PH;
    const double *fl = ph ? a.ph_pert : a.w;
    const BdyLeaf &lf = ph ? a.lph : a.lw;
    const double c1 = ld(g.c1f, k), c2 = ld(g.c2f, k);
    auto fls = [&](int jj, int ii) {
      const double mass = c1 * mu(jj, ii) + c2;
      return mass * ring_target(lf, zl, yl, xl, k, jj, ii) - mass * ld(fl, ix3(k, jj, ii, ny, nx));
    };
    val = div_msf(0.0 + relax_value(fls, side, j, i, yl, xl, a.fcx[b], a.gcx[b]), g.msfty, g.rmsfty, ix2(j, i, nx));
    double *t = (ph ? a.ph_tend : a.rw_tend) + ix3(k, j, i, ny, nx);
    *t = *t + val;
  } else {
    auto fls = [&](int jj, int ii) {
      return ring_target(a.lmu, 1, yl, xl, 0, jj, ii) - ld(a.mu_pert, ix2(jj, ii, nx));
    };
    val = 0.0 + relax_value(fls, side, j, i, yl, xl, a.fcx[b], a.gcx[b]);
    double *t = a.mu_tend + ix2(j, i, nx);
    *t = *t + val;
  }
}

// First-stage mu tendency: the base tendency (or zero) before the relax terms are added.
__global__ void k_mu_tend_init(Grid g, const double *base_mu, double *mu_tend) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const size_t c = ix2(j, i, g.nx);
  mu_tend[c] = (base_mu != nullptr) ? ld(base_mu, c) : 0.0;
}

// WRF zero_grad_bdy on w (core/acoustic.py:383-516, spec_zone 1): x threads
// over the ring-0 cells (S row, N row, then the W and E columns without the
// corners), blockIdx.y = level 0..nz.
__global__ void k_spec_w_zero_grad(Grid g, double *w, const double *w_save, const double *mut,
                                   const double *muts) {
  const int nx = g.nx, ny = g.ny;
  const int f = blockIdx.y;
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  int j, i, js, is;
  auto cl = [](int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); };
  if (e < nx) {
    j = 0; i = e; js = 1; is = cl(i, 1, nx - 2);
  } else if ((e -= nx) < nx) {
    j = ny - 1; i = e; js = ny - 2; is = cl(i, 1, nx - 2);
  } else if ((e -= nx) < ny - 2) {
    j = 1 + e; i = 0; js = cl(j, 1, ny - 2); is = 1;
  } else if ((e -= ny - 2) < ny - 2) {
    j = 1 + e; i = nx - 1; js = cl(j, 1, ny - 2); is = nx - 2;
  } else {
    return;
  }
  const double c1 = ld(g.c1f, f), c2 = ld(g.c2f, f);
  const size_t src2 = ix2(js, is, nx), dst2 = ix2(j, i, nx);
  const size_t src = ix3(f, js, is, ny, nx), dst = ix3(f, j, i, ny, nx);
  const double mc_s = c1 * ld(mut, src2) + c2, ms_s = c1 * ld(muts, src2) + c2;
  const double phys = (ld(g.msfty, src2) * w[src] + ld(w_save, src) * mc_s) / ms_s;
  const double mc_d = c1 * ld(mut, dst2) + c2, ms_d = c1 * ld(muts, dst2) + c2;
  w[dst] = div_msf(phys * ms_d - ld(w_save, dst) * mc_d, g.msfty, g.rmsfty, dst2);
}

}  // namespace wg
