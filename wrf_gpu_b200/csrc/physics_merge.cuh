// The RK1-fixed physics tendencies merged into every RK stage's tendencies
// (rk_addtend_dry, dynamics/core/rk_addtend_dry.py:490-546; WRF
// module_em.F:1711-1786), applied where _augment_large_step_tendencies
// applies it (operational_mode.py:3062-3075): after the advection, PGF and
// Coriolis terms and before the boundary-cadence relaxation.  Each field
// gets (tendf + [first stage] save * msf) coupled by its map factor:
//   u      += (ru_tendf + [rk1] u_save msfuy) / msfuy
//   v      += (rv_tendf + [rk1] v_save msfvx) * (1 / msfvx)
//   theta  += (t_tendf + [rk1] t_save) / msfty + (c1h mut + c2h) h_diabatic / msfty
//   mu     += mu_tendf
// (w is merged inside the w-face kernel, before pg_buoy_w is added, as the
// reference adds the merged tendency; ph has no consumer on this path).  A
// NULL leaf is the reference's zero leaf: its term adds an exact zero, so it
// is skipped.
#pragma once
#include "dycore_common.cuh"

namespace wg {

struct PhysArgs {
  const double *ru_tendf, *rv_tendf, *rw_tendf, *t_tendf, *mu_tendf, *h_diabatic;
  const double *u_save, *v_save, *w_save, *t_save;
  int rk1;  // the first RK stage (the boundary saves are added)
};

// mu tendency of every stage: the base tendency plus mu_tendf.
__global__ void k_phys_mu(Grid g, const double *base_mu, const double *mu_tendf, double *mu_tend) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const size_t c = ix2(j, i, g.nx);
  const double b = (base_mu != nullptr) ? ld(base_mu, c) : 0.0;
  mu_tend[c] = (mu_tendf != nullptr) ? b + ld(mu_tendf, c) : b;
}

// u, v and theta tendencies of one stage.  Index space (nx+1) x (ny+1) x nz.
__global__ void k_phys_merge(Grid g, PhysArgs a, const double *mu_total, double *u_tend, double *v_tend,
                             double *t_tend) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nxu = nx + 1, nyv = ny + 1;
  if (i > nx || j > ny) return;
  const bool us = a.rk1 && a.u_save != nullptr, vs = a.rk1 && a.v_save != nullptr;
  const bool ts = a.rk1 && a.t_save != nullptr;
  if (j < ny && (a.ru_tendf != nullptr || us)) {
    const size_t f2 = ix2(j, i, nxu), c = ix3(k, j, i, ny, nxu);
    double r = (a.ru_tendf != nullptr) ? ld(a.ru_tendf, c) : 0.0;
    if (us) r = r + ld(a.u_save, c) * ld(g.msfuy, f2);
    u_tend[c] = u_tend[c] + div_msf(r, g.msfuy, g.rmsfuy, f2);
  }
  if (i < nx && (a.rv_tendf != nullptr || vs)) {
    const size_t f2 = ix2(j, i, nx), c = ix3(k, j, i, nyv, nx);
    double r = (a.rv_tendf != nullptr) ? ld(a.rv_tendf, c) : 0.0;
    if (vs) r = r + ld(a.v_save, c) * ld(g.msfvx, f2);
    v_tend[c] = v_tend[c] + r * ld(g.rmsfvx, f2);
  }
  if (i < nx && j < ny && (a.t_tendf != nullptr || ts || a.h_diabatic != nullptr)) {
    const size_t c2 = ix2(j, i, nx), c = ix3(k, j, i, ny, nx);
    double th = t_tend[c];
    if (a.t_tendf != nullptr || ts) {
      double r = (a.t_tendf != nullptr) ? ld(a.t_tendf, c) : 0.0;
      if (ts) r = r + ld(a.t_save, c);
      th = th + div_msf(r, g.msfty, g.rmsfty, c2);
    }
    if (a.h_diabatic != nullptr) {
      const double mass_h = ld(g.c1h, k) * ld(mu_total, c2) + ld(g.c2h, k);
      th = th + div_msf(mass_h * ld(a.h_diabatic, c), g.msfty, g.rmsfty, c2);
    }
    t_tend[c] = th;
  }
}

}  // namespace wg
