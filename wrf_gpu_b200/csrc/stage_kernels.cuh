// Once-per-RK-stage kernels of the fp64 dycore step: transport velocities,
// diagnostics, flux-form advection, large-step PGF/Coriolis, small_step_prep,
// pg_buoy_w, rhs_ph, calc_coef_w and the step-0 calc_p_rho.
//
// Every expression keeps the operation order of the reference JAX code it
// cites; the translation unit is compiled with -fmad=false so float64 results
// track the reference's unfused arithmetic.
#pragma once
#include "dycore_common.cuh"

namespace wg {

// ---------------------------------------------------------------------------
// 2-D stage masses: small_step_prep (core/small_step_prep.py:259-274, 75-86)
// plus the acoustic mass work arrays (operational_mode.py:2052-2060).
// Index space (ny+1) x (nx+1).
// ---------------------------------------------------------------------------
struct Mass2D {
  double *mub, *mut, *muts0, *mu_work0;   // (ny, nx)
  double *muu, *muus;                     // (ny, nx+1) edge-padded face averages of mut / muts
  double *muv, *muvs;                     // (ny+1, nx)
  double *mu_ac, *muts_ac, *muave_ac;     // acoustic work (ny, nx)
};

__device__ __forceinline__ void mut_muts_at(const StateR &s, const double *ref_mu_pert, int rk_step, size_t c,
                                            double &mut, double &muts) {
  double mub = ld(s.mu_total, c) - ld(s.mu_pert, c);
  double mu_cur = ld(s.mu_pert, c);
  double mu_work = (rk_step == 1) ? 0.0 : ld(ref_mu_pert, c) - mu_cur;
  mut = mub + mu_cur;
  muts = mut + mu_work;
}

__global__ void k_mass2d(Grid g, StateR s, const double *ref_mu_pert, int rk_step, Mass2D o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny;
  if (i > nx || j > ny) return;
  if (j < ny && i < nx) {
    size_t c = ix2(j, i, nx);
    double mub = ld(s.mu_total, c) - ld(s.mu_pert, c);
    double mu_cur = ld(s.mu_pert, c);
    double mu_work = (rk_step == 1) ? 0.0 : ld(ref_mu_pert, c) - mu_cur;
    double mut = mub + mu_cur;
    double muts = mut + mu_work;
    o.mub[c] = mub;
    o.mut[c] = mut;
    o.muts0[c] = muts;
    o.mu_work0[c] = mu_work;
    o.mu_ac[c] = mu_cur + mu_work;
    o.muts_ac[c] = muts;
    o.muave_ac[c] = 0.0;
  }
  if (j < ny) {
    double mut_l, muts_l, mut_r, muts_r;
    if (i == 0) {
      mut_muts_at(s, ref_mu_pert, rk_step, ix2(j, 0, nx), mut_l, muts_l);
      o.muu[ix2(j, i, nx + 1)] = mut_l;
      o.muus[ix2(j, i, nx + 1)] = muts_l;
    } else if (i == nx) {
      mut_muts_at(s, ref_mu_pert, rk_step, ix2(j, nx - 1, nx), mut_r, muts_r);
      o.muu[ix2(j, i, nx + 1)] = mut_r;
      o.muus[ix2(j, i, nx + 1)] = muts_r;
    } else {
      mut_muts_at(s, ref_mu_pert, rk_step, ix2(j, i - 1, nx), mut_l, muts_l);
      mut_muts_at(s, ref_mu_pert, rk_step, ix2(j, i, nx), mut_r, muts_r);
      o.muu[ix2(j, i, nx + 1)] = 0.5 * (mut_l + mut_r);
      o.muus[ix2(j, i, nx + 1)] = 0.5 * (muts_l + muts_r);
    }
  }
  if (i < nx) {
    double mut_s, muts_s, mut_n, muts_n;
    if (j == 0) {
      mut_muts_at(s, ref_mu_pert, rk_step, ix2(0, i, nx), mut_s, muts_s);
      o.muv[ix2(j, i, nx)] = mut_s;
      o.muvs[ix2(j, i, nx)] = muts_s;
    } else if (j == ny) {
      mut_muts_at(s, ref_mu_pert, rk_step, ix2(ny - 1, i, nx), mut_n, muts_n);
      o.muv[ix2(j, i, nx)] = mut_n;
      o.muvs[ix2(j, i, nx)] = muts_n;
    } else {
      mut_muts_at(s, ref_mu_pert, rk_step, ix2(j - 1, i, nx), mut_s, muts_s);
      mut_muts_at(s, ref_mu_pert, rk_step, ix2(j, i, nx), mut_n, muts_n);
      o.muv[ix2(j, i, nx)] = 0.5 * (mut_s + mut_n);
      o.muvs[ix2(j, i, nx)] = 0.5 * (muts_s + muts_n);
    }
  }
}

// ---------------------------------------------------------------------------
// Transport velocities (flux_advection.py:394-470 couple_velocities_periodic)
// and, for specified/nested domains, the edge-faithful stage omega
// (flux_advection.py:180-232 stage_omega_specified).  One thread per column.
// ---------------------------------------------------------------------------
__global__ void k_transport(Grid g, const double *u, const double *v, const double *mu_total, double *ru, double *rv,
                            double *rom, double *ww_spec) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  const int ip = wrp(i + 1, nx), im = wrp(i - 1, nx), jp = wrp(j + 1, ny), jm = wrp(j - 1, ny);
  const double mu_c = ld(mu_total, ix2(j, i, nx));
  const double muu_i = 0.5 * (mu_c + ld(mu_total, ix2(j, im, nx)));
  const double muu_ip = 0.5 * (ld(mu_total, ix2(j, ip, nx)) + mu_c);
  const double muv_j = 0.5 * (mu_c + ld(mu_total, ix2(jm, i, nx)));
  const double muv_jp = 0.5 * (ld(mu_total, ix2(jp, i, nx)) + mu_c);
  const double msfuy_i = ld(g.msfuy, ix2(j, i, nx + 1)), msfuy_ip = ld(g.msfuy, ix2(j, ip, nx + 1));
  const double msfvx_j = ld(g.msfvx, ix2(j, i, nx)), msfvx_jp = ld(g.msfvx, ix2(jp, i, nx));
  const double msftx = ld(g.msftx, ix2(j, i, nx));
  double dmdt = 0.0;
  for (int k = 0; k < nz; ++k) {
    const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
    double ru_i = (c1 * muu_i + c2) * ld(u, ix3(k, j, i, ny, nx + 1)) / msfuy_i;
    double ru_ip = (c1 * muu_ip + c2) * ld(u, ix3(k, j, ip, ny, nx + 1)) / msfuy_ip;
    double rv_j = (c1 * muv_j + c2) * ld(v, ix3(k, j, i, ny + 1, nx)) / msfvx_j;
    double rv_jp = (c1 * muv_jp + c2) * ld(v, ix3(k, jp, i, ny + 1, nx)) / msfvx_jp;
    double divv = ld(g.dnw, k) * msftx * (g.rdx * (ru_ip - ru_i) + g.rdy * (rv_jp - rv_j));
    dmdt = (k == 0) ? divv : dmdt + divv;
    ru[ix3(k, j, i, ny, nx)] = ru_i;
    rv[ix3(k, j, i, ny, nx)] = rv_j;
  }
  double cum = 0.0;
  rom[ix3(0, j, i, ny, nx)] = 0.0;
  for (int k = 0; k < nz - 1; ++k) {
    const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
    double ru_i = (c1 * muu_i + c2) * ld(u, ix3(k, j, i, ny, nx + 1)) / msfuy_i;
    double ru_ip = (c1 * muu_ip + c2) * ld(u, ix3(k, j, ip, ny, nx + 1)) / msfuy_ip;
    double rv_j = (c1 * muv_j + c2) * ld(v, ix3(k, j, i, ny + 1, nx)) / msfvx_j;
    double rv_jp = (c1 * muv_jp + c2) * ld(v, ix3(k, jp, i, ny + 1, nx)) / msfvx_jp;
    double divv = ld(g.dnw, k) * msftx * (g.rdx * (ru_ip - ru_i) + g.rdy * (rv_jp - rv_j));
    double inc = -(ld(g.dnw, k) * c1 * dmdt) - divv;
    cum = (k == 0) ? inc : cum + inc;
    rom[ix3(k + 1, j, i, ny, nx)] = cum;
  }
  rom[ix3(nz, j, i, ny, nx)] = 0.0;

  if (ww_spec != nullptr) {
    // stage_omega_specified: edge-padded face masses, full staggered faces.
    const double mu_w = (i == 0) ? mu_c : ld(mu_total, ix2(j, i - 1, nx));
    const double muu_s_i = 0.5 * (mu_c + mu_w);
    const double muu_s_ip = (i + 1 == nx) ? mu_c : 0.5 * (ld(mu_total, ix2(j, i + 1, nx)) + mu_c);
    const double mu_s = (j == 0) ? mu_c : ld(mu_total, ix2(j - 1, i, nx));
    const double muv_s_j = 0.5 * (mu_c + mu_s);
    const double muv_s_jp = (j + 1 == ny) ? mu_c : 0.5 * (ld(mu_total, ix2(j + 1, i, nx)) + mu_c);
    const double fuy_i = ld(g.msfuy, ix2(j, i, nx + 1)), fuy_ip = ld(g.msfuy, ix2(j, i + 1, nx + 1));
    const double fvx_j = ld(g.msfvx, ix2(j, i, nx)), fvx_jp = ld(g.msfvx, ix2(j + 1, i, nx));
    double dm = 0.0;
    for (int k = 0; k < nz; ++k) {
      const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
      double a0 = (c1 * muu_s_i + c2) * ld(u, ix3(k, j, i, ny, nx + 1)) / fuy_i;
      double a1 = (c1 * muu_s_ip + c2) * ld(u, ix3(k, j, i + 1, ny, nx + 1)) / fuy_ip;
      double b0 = (c1 * muv_s_j + c2) * ld(v, ix3(k, j, i, ny + 1, nx)) / fvx_j;
      double b1 = (c1 * muv_s_jp + c2) * ld(v, ix3(k, j + 1, i, ny + 1, nx)) / fvx_jp;
      double divv = msftx * ld(g.dnw, k) * (g.rdx * (a1 - a0) + g.rdy * (b1 - b0));
      dm = (k == 0) ? divv : dm + divv;
    }
    double cm = 0.0;
    ww_spec[ix3(0, j, i, ny, nx)] = 0.0;
    for (int k = 0; k < nz - 1; ++k) {
      const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
      double a0 = (c1 * muu_s_i + c2) * ld(u, ix3(k, j, i, ny, nx + 1)) / fuy_i;
      double a1 = (c1 * muu_s_ip + c2) * ld(u, ix3(k, j, i + 1, ny, nx + 1)) / fuy_ip;
      double b0 = (c1 * muv_s_j + c2) * ld(v, ix3(k, j, i, ny + 1, nx)) / fvx_j;
      double b1 = (c1 * muv_s_jp + c2) * ld(v, ix3(k, j + 1, i, ny + 1, nx)) / fvx_jp;
      double divv = msftx * ld(g.dnw, k) * (g.rdx * (a1 - a0) + g.rdy * (b1 - b0));
      double inc = -(ld(g.dnw, k) * c1 * dm) - divv;
      cm = (k == 0) ? inc : cm + inc;
      ww_spec[ix3(k + 1, j, i, ny, nx)] = cm;
    }
    ww_spec[ix3(nz, j, i, ny, nx)] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// Per-cell diagnostics for the stage (mass points):
//   alt_raw = EOS(theta, p_total)            (rk_addtend_dry.py:171-173)
//   alt     = max(alt_raw, 0.1)              (small_step_prep.py:334)
//   pb      = p_total - p'                   (small_step_prep.py:335)
//   c2a     = cpovcv*(pb+p')/alt             (small_step_prep.py:335)
//   qtot    = qv+qc+qr+qi+qs+qg              (acoustic_wrf.py:316)
//   al_ls   = large-step al                  (rk_addtend_dry.py:186-224)
//   php_ls  = 0.5*(pht(k)+pht(k+1))          (rk_addtend_dry.py:227-228)
//   php     = stage-constant php             (small_step_prep.py:350-352)
// ---------------------------------------------------------------------------
struct Diag {
  double *alt_raw, *alt, *pb, *c2a, *qtot, *al_ls, *php_ls, *php;
};

__global__ void k_diag(Grid g, StateR s, int hyps, Diag o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny;
  if (i >= nx || j >= ny) return;
  const size_t c = ix3(k, j, i, ny, nx);
  const size_t f0 = c, f1 = ix3(k + 1, j, i, ny, nx);
  const size_t c2d = ix2(j, i, nx);
  const double theta = ld(s.theta, c), pt = ld(s.p_total, c), pp = ld(s.p_pert, c);
  const double alt_raw = inv_density(theta, pt);
  const double alt = dmax(alt_raw, MIN_ACOUSTIC_ALT);
  const double pb = pt - pp;
  o.alt_raw[c] = alt_raw;
  o.alt[c] = alt;
  o.pb[c] = pb;
  o.c2a[c] = CPOVCV * (pb + pp) / alt;
  double qt = 0.0;
  if (s.q[0] != nullptr) {
    qt = ld(s.q[0], c) + ld(s.q[1], c) + ld(s.q[2], c) + ld(s.q[3], c) + ld(s.q[4], c) + ld(s.q[5], c);
  }
  o.qtot[c] = qt;
  const double ph0 = ld(s.ph_pert, f0), ph1 = ld(s.ph_pert, f1);
  const double phb0 = ld(s.ph_total, f0) - ph0, phb1 = ld(s.ph_total, f1) - ph1;
  const double mu_total = ld(s.mu_total, c2d), mu_pert = ld(s.mu_pert, c2d);
  const double mub = mu_total - mu_pert;
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k), rdnw = ld(g.rdnw, k);
  double al;
  if (hyps == 2) {
    const double c3f0 = ld(g.c3f, k), c3f1 = ld(g.c3f, k + 1), c4f0 = ld(g.c4f, k), c4f1 = ld(g.c4f, k + 1);
    const double c3h = ld(g.c3h, k), c4h = ld(g.c4h, k);
    const double dph_tot = (phb1 + ph1) - (phb0 + ph0);
    double pfu = c3f1 * mu_total + c4f1 + g.p_top;
    double pfd = c3f0 * mu_total + c4f0 + g.p_top;
    double phm = c3h * mu_total + c4h + g.p_top;
    double a1 = dph_tot / phm / log(pfd / pfu);
    pfu = c3f1 * mub + c4f1 + g.p_top;
    pfd = c3f0 * mub + c4f0 + g.p_top;
    phm = c3h * mub + c4h + g.p_top;
    double a2 = (phb1 - phb0) / phm / log(pfd / pfu);
    al = a1 - a2;
  } else {
    const double mass_base = c1 * mub + c2;
    const double alb = -rdnw * (phb1 - phb0) / safe12(mass_base);
    const double muts = mu_total + mu_pert;
    const double mass_t = c1 * muts + c2;
    const double mu_term = c1 * mu_pert;
    al = -(alb * mu_term + rdnw * (ph1 - ph0)) / safe12(mass_t);
  }
  o.al_ls[c] = al;
  const double pht0 = phb0 + ph0, pht1 = phb1 + ph1;
  o.php_ls[c] = 0.5 * (pht0 + pht1);
  o.php[c] = 0.5 * (phb0 + phb1 + ph0 + ph1);
}

// dpn at face m (large-step form, rk_addtend_dry.py:290-301).  ps(m) is the
// mass-level pair sum.
template <typename PS>
__device__ __forceinline__ double dpn_large(const Grid &g, int m, int top_lid, PS ps) {
  const int nz = g.nz;
  if (m == 0) return 0.5 * (g.cf1 * ps(0) + g.cf2 * ps(1) + g.cf3 * ps(2));
  if (m < nz) return 0.5 * (ld(g.fnm, m) * ps(m) + ld(g.fnp, m) * ps(m - 1));
  if (top_lid) return 0.5 * (g.cfn * ps(nz - 1) + g.cfn1 * ps(nz - 2));
  return 0.0;
}

// dpn at face m (acoustic form, core/acoustic.py:563-580).
template <typename PS>
__device__ __forceinline__ double dpn_acoustic(const Grid &g, int m, int top_lid, PS ps) {
  const int nz = g.nz;
  if (m == 0) return 0.5 * (g.cf1 * ps(0) + g.cf2 * ps(1) + g.cf3 * ps(2));
  if (m < nz) return 0.5 * (ld(g.fnm, m) * ps(m) + ld(g.fnp, m) * ps(m - 1));
  if (top_lid) return 0.5 * (g.cf1 * ps(nz - 1) + g.cf2 * ps(nz - 2) + g.cf3 * ps(nz - 3));
  return 0.0;
}

// Order-3 vertical flux of a mass-level field at face m (flux_advection.py:1362-1407
// for u/v, :534-562 for scalars; both use -sign(vel)).
template <typename Q>
__device__ __forceinline__ double vflux3_at(const Grid &g, int m, double romq, Q q) {
  const int nz = g.nz;
  if (m <= 0 || m >= nz) return 0.0;
  if (m == 1) return romq * (ld(g.fnm, 1) * q(1) + ld(g.fnp, 1) * q(0));
  if (m == nz - 1) return romq * (ld(g.fnm, nz - 1) * q(nz - 1) + ld(g.fnp, nz - 1) * q(nz - 2));
  return flux3v(q(m - 2), q(m - 1), q(m), q(m + 1), romq);
}

// ---------------------------------------------------------------------------
// u faces: advect_u_flux (flux_advection.py:1131-1202) + base tendency,
// large-step PGF (rk_addtend_dry.py:303-317, 344-346), Coriolis
// (rk_addtend_dry.py:405-446), small_step_prep u_work (small_step_prep.py:319).
// ---------------------------------------------------------------------------
struct UFaceOut {
  double *u_tend, *u_w, *cqu;
};

__global__ void k_uface(Grid g, StateR s, StateR ref, const double *ru, const double *rv, const double *rom,
                        Diag d, const double *muu, const double *muus, const double *base_u, int top_lid,
                        int run_boundary, UFaceOut o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i > nx || j >= ny) return;
  const int nxu = nx + 1;
  const size_t cu = ix3(k, j, i, ny, nxu);
  // ---- advection on the periodic collapsed faces ----
  const int ii = (i == nx) ? 0 : i;
  auto uf = [&](int kk, int jj, int mm) { return ld(s.u, ix3(kk, wrp(jj, ny), wrp(mm, nx), ny, nxu)); };
  auto fqx = [&](int m) {
    int rm = wrp(m, nx);
    double vel = 0.5 * (ld(ru, ix3(k, j, rm, ny, nx)) + ld(ru, ix3(k, j, wrp(rm - 1, nx), ny, nx)));
    return vel * flux5(uf(k, j, rm - 3), uf(k, j, rm - 2), uf(k, j, rm - 1), uf(k, j, rm), uf(k, j, rm + 1),
                       uf(k, j, rm + 2), vel);
  };
  const double msfux_c = ld(g.msfux, ix2(j, ii, nxu));
  double tend = -msfux_c * g.rdx * (fqx(ii + 1) - fqx(ii));
  if (ny > 1) {
    auto fqy = [&](int n) {
      int rn = wrp(n, ny);
      double vel = 0.5 * (ld(rv, ix3(k, rn, ii, ny, nx)) + ld(rv, ix3(k, rn, wrp(ii - 1, nx), ny, nx)));
      return vel * flux5(uf(k, rn - 3, ii), uf(k, rn - 2, ii), uf(k, rn - 1, ii), uf(k, rn, ii), uf(k, rn + 1, ii),
                         uf(k, rn + 2, ii), vel);
    };
    tend = tend - msfux_c * g.rdy * (fqy(j + 1) - fqy(j));
  }
  {
    auto romq = [&](int m) {
      return 0.5 * (ld(rom, ix3(m, j, ii, ny, nx)) + ld(rom, ix3(m, j, wrp(ii - 1, nx), ny, nx)));
    };
    auto q = [&](int kk) { return ld(s.u, ix3(kk, j, ii, ny, nxu)); };
    double v1 = (k + 1 <= nz - 1) ? vflux3_at(g, k + 1, romq(k + 1), q) : 0.0;
    double v0 = (k >= 1) ? vflux3_at(g, k, romq(k), q) : 0.0;
    tend = tend + (-ld(g.rdnw, k)) * (v1 - v0);
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
  // ---- large-step horizontal PGF (edge-padded face pairs) ----
  {
    auto P = [&](const double *a, int kk, int ic) { return ld(a, ix3(kk, j, ic, ny, nx)); };
    const double ph_term = (P(s.ph_pert, k + 1, r) - P(s.ph_pert, k + 1, l)) + (P(s.ph_pert, k, r) - P(s.ph_pert, k, l));
    const double p_term = (P(d.alt_raw, k, l) + P(d.alt_raw, k, r)) * (P(s.p_pert, k, r) - P(s.p_pert, k, l));
    const double pb_term = (P(d.al_ls, k, l) + P(d.al_ls, k, r)) * (P(d.pb, k, r) - P(d.pb, k, l));
    const double mp_l = ld(s.mu_pert, ix2(j, l, nx)), mp_r = ld(s.mu_pert, ix2(j, r, nx));
    const double mt_l = (ld(s.mu_total, ix2(j, l, nx)) - mp_l) + mp_l;
    const double mt_r = (ld(s.mu_total, ix2(j, r, nx)) - mp_r) + mp_r;
    const double mass_u = c1 * (0.5 * (mt_l + mt_r)) + c2;
    const double msf_u = ld(g.msfux, ix2(j, i, nxu)) / ld(g.msfuy, ix2(j, i, nxu));
    double dpx = msf_u * 0.5 * g.rdx * mass_u * (ph_term + p_term + pb_term);
    auto ps = [&](int m) { return P(s.p_pert, m, l) + P(s.p_pert, m, r); };
    const double bracket = ld(g.rdnw, k) * (dpn_large(g, k + 1, top_lid, ps) - dpn_large(g, k, top_lid, ps)) -
                           0.5 * (c1 * (mp_l + mp_r));
    dpx = dpx + msf_u * g.rdx * (P(d.php_ls, k, r) - P(d.php_ls, k, l)) * bracket;
    const double cqu = 1.0 / (1.0 + 0.5 * (P(d.qtot, k, l) + P(d.qtot, k, r)));
    u_t = u_t + (-cqu) * dpx;
    o.cqu[cu] = cqu;
  }
  // ---- Coriolis (rk_addtend_dry.py:405-446) ----
  {
    auto mu2 = [&](int jj, int ic) { return ld(s.mu_total, ix2(jj, ic, nx)); };
    auto rvq = [&](int jv, int ic) {  // coupled v at v-face (jv, ic)
      const int js = (jv == 0) ? 0 : jv - 1, jn = (jv == ny) ? ny - 1 : jv;
      const double muv_c = 0.5 * (mu2(js, ic) + mu2(jn, ic));
      return ld(s.v, ix3(k, jv, ic, ny + 1, nx)) * (c1 * muv_c + c2) / ld(g.msfvx, ix2(jv, ic, nx));
    };
    auto rwq = [&](int kf, int ic) {
      return ld(s.w, ix3(kf, j, ic, ny, nx)) * (ld(g.c1f, kf) * mu2(j, ic) + ld(g.c2f, kf)) /
             ld(g.msfty, ix2(j, ic, nx));
    };
    const double rv_quad = 0.25 * (rvq(j, l) + rvq(j, r) + rvq(j + 1, l) + rvq(j + 1, r));
    const double f_u = 0.5 * (ld(g.f, ix2(j, l, nx)) + ld(g.f, ix2(j, r, nx)));
    const double e_u = 0.5 * (ld(g.e, ix2(j, l, nx)) + ld(g.e, ix2(j, r, nx)));
    const double cosa_u = 0.5 * (ld(g.cosa, ix2(j, l, nx)) + ld(g.cosa, ix2(j, r, nx)));
    const double msf_u = ld(g.msfux, ix2(j, i, nxu)) / ld(g.msfuy, ix2(j, i, nxu));
    double ru_cor = msf_u * f_u * rv_quad;
    const double rw_quad = 0.25 * (rwq(k, l) + rwq(k + 1, l) + rwq(k, r) + rwq(k + 1, r));
    ru_cor = ru_cor - e_u * cosa_u * rw_quad;
    if (run_boundary && (i == 0 || i == nx)) ru_cor = ru_cor * 0.0;
    u_t = u_t + ru_cor;
  }
  o.u_tend[cu] = u_t;
  // ---- small_step_prep u_work ----
  const size_t f2 = ix2(j, i, nxu);
  const double mass_ref = c1 * ld(muus, f2) + c2;
  const double mass_cur = c1 * ld(muu, f2) + c2;
  o.u_w[cu] = (mass_ref * ld(ref.u, cu) - mass_cur * ld(s.u, cu)) / ld(g.msfuy, f2);
}

// ---------------------------------------------------------------------------
// v faces: advect_v_flux (flux_advection.py:1205-1274) + base, PGF
// (rk_addtend_dry.py:320-341, 344-346), Coriolis (:448-466), v_work
// (small_step_prep.py:320).
// ---------------------------------------------------------------------------
struct VFaceOut {
  double *v_tend, *v_w, *cqv;
};

__global__ void k_vface(Grid g, StateR s, StateR ref, const double *ru, const double *rv, const double *rom,
                        Diag d, const double *muv, const double *muvs, const double *base_v, int top_lid,
                        int run_boundary, VFaceOut o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny;
  if (i >= nx || j > ny) return;
  const int nyv = ny + 1;
  const size_t cv = ix3(k, j, i, nyv, nx);
  const int jj = (j == ny) ? 0 : j;
  auto vf = [&](int kk, int jv, int ic) { return ld(s.v, ix3(kk, wrp(jv, ny), wrp(ic, nx), nyv, nx)); };
  const double msfvy_c = ld(g.msfvy, ix2(jj, i, nx));
  const double msfvx_c = ld(g.msfvx, ix2(jj, i, nx));
  auto fqx = [&](int m) {
    int rm = wrp(m, nx);
    double vel = 0.5 * (ld(ru, ix3(k, jj, rm, ny, nx)) + ld(ru, ix3(k, wrp(jj - 1, ny), rm, ny, nx)));
    return vel * flux5(vf(k, jj, rm - 3), vf(k, jj, rm - 2), vf(k, jj, rm - 1), vf(k, jj, rm), vf(k, jj, rm + 1),
                       vf(k, jj, rm + 2), vel);
  };
  double tend = -msfvy_c * g.rdx * (fqx(i + 1) - fqx(i));
  auto fqy = [&](int n) {
    int rn = wrp(n, ny);
    double vel = 0.5 * (ld(rv, ix3(k, rn, i, ny, nx)) + ld(rv, ix3(k, wrp(rn - 1, ny), i, ny, nx)));
    return vel * flux5(vf(k, rn - 3, i), vf(k, rn - 2, i), vf(k, rn - 1, i), vf(k, rn, i), vf(k, rn + 1, i),
                       vf(k, rn + 2, i), vel);
  };
  tend = tend - msfvy_c * g.rdy * (fqy(jj + 1) - fqy(jj));
  {
    auto romq = [&](int m) {
      return 0.5 * (ld(rom, ix3(m, jj, i, ny, nx)) + ld(rom, ix3(m, wrp(jj - 1, ny), i, ny, nx)));
    };
    auto q = [&](int kk) { return ld(s.v, ix3(kk, jj, i, nyv, nx)); };
    const int nz = g.nz;
    double v1 = (k + 1 <= nz - 1) ? vflux3_at(g, k + 1, romq(k + 1), q) : 0.0;
    double v0 = (k >= 1) ? vflux3_at(g, k, romq(k), q) : 0.0;
    tend = tend + (msfvy_c / msfvx_c) * ((-ld(g.rdnw, k)) * (v1 - v0));
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
    const double msf_v = ld(g.msfvy, ix2(j, i, nx)) / ld(g.msfvx, ix2(j, i, nx));
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
    auto ruq = [&](int jc, int iu) {  // coupled u at u-face (jc, iu)
      const int il = (iu == 0) ? 0 : iu - 1, ir = (iu == nx) ? nx - 1 : iu;
      const double muu_c = 0.5 * (mu2(jc, il) + mu2(jc, ir));
      return ld(s.u, ix3(k, jc, iu, ny, nx + 1)) * (c1 * muu_c + c2) / ld(g.msfuy, ix2(jc, iu, nx + 1));
    };
    auto rwq = [&](int kf, int jc) {
      return ld(s.w, ix3(kf, jc, i, ny, nx)) * (ld(g.c1f, kf) * mu2(jc, i) + ld(g.c2f, kf)) /
             ld(g.msfty, ix2(jc, i, nx));
    };
    const double ru_quad = 0.25 * (ruq(sj, i) + ruq(sj, i + 1) + ruq(nj, i) + ruq(nj, i + 1));
    const double f_v = 0.5 * (ld(g.f, ix2(sj, i, nx)) + ld(g.f, ix2(nj, i, nx)));
    const double e_v = 0.5 * (ld(g.e, ix2(sj, i, nx)) + ld(g.e, ix2(nj, i, nx)));
    const double sina_v = 0.5 * (ld(g.sina, ix2(sj, i, nx)) + ld(g.sina, ix2(nj, i, nx)));
    const double msf_v = ld(g.msfvy, ix2(j, i, nx)) / ld(g.msfvx, ix2(j, i, nx));
    double rv_cor = -msf_v * f_v * ru_quad;
    const double rw_quad = 0.25 * (rwq(k, sj) + rwq(k + 1, sj) + rwq(k, nj) + rwq(k + 1, nj));
    rv_cor = rv_cor + msf_v * e_v * sina_v * rw_quad;
    if (run_boundary && (j == 0 || j == ny)) rv_cor = rv_cor * 0.0;
    v_t = v_t + rv_cor;
  }
  o.v_tend[cv] = v_t;
  const size_t f2 = ix2(j, i, nx);
  const double mass_ref = c1 * ld(muvs, f2) + c2;
  const double mass_cur = c1 * ld(muv, f2) + c2;
  o.v_w[cv] = (mass_ref * ld(ref.v, cv) - mass_cur * ld(s.v, cv)) / ld(g.msfvx, f2);
}

// ---------------------------------------------------------------------------
// Plain h5/v3 scalar advection tendency at cell (k, j, i)
// (flux_advection.py:482-568).  q(kk, jj, ii) returns the advected value.
// ---------------------------------------------------------------------------
template <typename Q>
__device__ __forceinline__ double scalar_adv(const Grid &g, int k, int j, int i, const double *ru, const double *rv,
                                             const double *rom, Q q) {
  const int nx = g.nx, ny = g.ny;
  auto fqx = [&](int m) {
    int rm = wrp(m, nx);
    double vel = ld(ru, ix3(k, j, rm, ny, nx));
    return vel * flux5(q(k, j, rm - 3), q(k, j, rm - 2), q(k, j, rm - 1), q(k, j, rm), q(k, j, rm + 1),
                       q(k, j, rm + 2), vel);
  };
  auto fqy = [&](int n) {
    int rn = wrp(n, ny);
    double vel = ld(rv, ix3(k, rn, i, ny, nx));
    return vel * flux5(q(k, rn - 3, i), q(k, rn - 2, i), q(k, rn - 1, i), q(k, rn, i), q(k, rn + 1, i),
                       q(k, rn + 2, i), vel);
  };
  const double msftx = ld(g.msftx, ix2(j, i, nx));
  double tend = -msftx * g.rdx * (fqx(i + 1) - fqx(i));
  tend = tend - msftx * g.rdy * (fqy(j + 1) - fqy(j));
  auto qc = [&](int kk) { return q(kk, j, i); };
  const int nz = g.nz;
  double v1 = (k + 1 <= nz - 1) ? vflux3_at(g, k + 1, ld(rom, ix3(k + 1, j, i, ny, nx)), qc) : 0.0;
  double v0 = (k >= 1) ? vflux3_at(g, k, ld(rom, ix3(k, j, i, ny, nx)), qc) : 0.0;
  return tend - ld(g.rdnw, k) * (v1 - v0);
}

// Mass-point stage kernel: theta tendency (plain path), moisture tendencies
// (plain path), theta_work (small_step_prep.py:321).
struct MassOut {
  double *t_tend, *theta_w;
  double *q_tend[6];
};

__global__ void k_mass(Grid g, StateR s, StateR ref, const double *ru, const double *rv, const double *rom,
                       const double *mut, const double *muts0, const double *base_theta, int theta_plain,
                       int moist_plain, MassOut o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny;
  if (i >= nx || j >= ny) return;
  const size_t c = ix3(k, j, i, ny, nx);
  const size_t c2d = ix2(j, i, nx);
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  if (theta_plain) {
    auto q = [&](int kk, int jj, int ii2) { return ld(s.theta, ix3(kk, wrp(jj, ny), wrp(ii2, nx), ny, nx)) - T0; };
    double adv = scalar_adv(g, k, j, i, ru, rv, rom, q);
    if (base_theta != nullptr) {
      const double mass_h = c1 * ld(s.mu_total, c2d) + c2;
      o.t_tend[c] = ld(base_theta, c) * mass_h + adv;
    } else {
      o.t_tend[c] = adv;
    }
  }
  if (moist_plain) {
    for (int sp = 0; sp < 6; ++sp) {
      const double *qa = s.q[sp];
      auto q = [&](int kk, int jj, int ii2) { return ld(qa, ix3(kk, wrp(jj, ny), wrp(ii2, nx), ny, nx)); };
      o.q_tend[sp][c] = scalar_adv(g, k, j, i, ru, rv, rom, q);
    }
  }
  const double mass_ref = c1 * ld(muts0, c2d) + c2;
  const double mass_cur = c1 * ld(mut, c2d) + c2;
  o.theta_w[c] = mass_ref * (ld(ref.theta, c) - T0) - mass_cur * (ld(s.theta, c) - T0);
}

// ---------------------------------------------------------------------------
// Positive-definite / monotonic limited scalar advection
// (flux_advection.py:736-1000), periodic path.  Two passes: k_lim_scale
// computes the per-cell limiter scale(s), k_lim_tend the tendency.
// ---------------------------------------------------------------------------
struct LimArgs {
  const double *ru, *rv, *rom;
  const double *mut;     // current total dry mass (ny, nx)
  const double *mu_old;  // start-of-step total dry mass (ny, nx)
  double dt;
  int opt;               // 1 PD, 2 mono
  double offset;         // subtracted from both fields (300 for theta, 0 for q)
  // Per-launch constants of the upwind fluxes (set by set_lim_constants):
  // dx = 1/rdx and dy = 1/rdy as the reference forms them, their correctly
  // rounded reciprocals (divisors for div_rcp), 1/dt, dx/dt and dy/dt.
  double dxl, dyl, rdxl, rdyl, rdt, dxl_dt, dyl_dt;
};

inline void set_lim_constants(LimArgs &a, double rdx, double rdy) {
  a.dxl = 1.0 / rdx;
  a.dyl = 1.0 / rdy;
  a.rdxl = 1.0 / a.dxl;
  a.rdyl = 1.0 / a.dyl;
  a.rdt = 1.0 / a.dt;
  a.dxl_dt = a.dxl / a.dt;
  a.dyl_dt = a.dyl / a.dt;
}

struct CellFluxes {
  double lx0, lx1, ly0, ly1, lz0, lz1;  // low-order fluxes at the 6 faces
  double ax0, ax1, ay0, ay1, az0, az1;  // antidiffusive fluxes
};

template <typename QF, typename QO>
__device__ __forceinline__ void cell_fluxes(const Grid &g, const LimArgs &a, int k, int j, int i, QF qf, QO qo,
                                            CellFluxes &cf) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double dx = 1.0 / g.rdx, dy = 1.0 / g.rdy;
  auto mut2 = [&](int jj, int ii2) { return ld(a.mut, ix2(wrp(jj, ny), wrp(ii2, nx), nx)); };
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  auto upw = [&](double fo_m1, double fo_0, double vel, double mu_face, double dxy) {
    double cr = vel * a.dt / dxy / mu_face;
    double ab = fabs(cr);
    return mu_face * (dxy / a.dt) * (0.5 * dmin(1.0, cr + ab) * fo_m1 + 0.5 * dmax(-1.0, cr - ab) * fo_0);
  };
  // x faces m = i, i+1
  auto xf = [&](int m, double &lo, double &an) {
    int rm = wrp(m, nx);
    double vel = ld(a.ru, ix3(k, j, rm, ny, nx));
    double muu = 0.5 * (mut2(j, rm) + mut2(j, rm - 1));
    double mu_u = c1 * muu + c2;
    lo = upw(qo(k, j, rm - 1), qo(k, j, rm), vel, mu_u, dx);
    double hi = vel * flux5(qf(k, j, rm - 3), qf(k, j, rm - 2), qf(k, j, rm - 1), qf(k, j, rm), qf(k, j, rm + 1),
                            qf(k, j, rm + 2), vel);
    an = hi - lo;
  };
  auto yf = [&](int n, double &lo, double &an) {
    int rn = wrp(n, ny);
    double vel = ld(a.rv, ix3(k, rn, i, ny, nx));
    double muv = 0.5 * (mut2(rn, i) + mut2(rn - 1, i));
    double mu_v = c1 * muv + c2;
    lo = upw(qo(k, rn - 1, i), qo(k, rn, i), vel, mu_v, dy);
    double hi = vel * flux5(qf(k, rn - 3, i), qf(k, rn - 2, i), qf(k, rn - 1, i), qf(k, rn, i), qf(k, rn + 1, i),
                            qf(k, rn + 2, i), vel);
    an = hi - lo;
  };
  auto zf = [&](int m, double &lo, double &an) {
    if (m <= 0 || m >= nz) {
      lo = 0.0;
      an = 0.0;
      return;
    }
    double romv = ld(a.rom, ix3(m, j, i, ny, nx));
    double mt = ld(a.mut, ix2(j, i, nx));
    double muh_m = ld(g.c1h, m) * mt + ld(g.c2h, m);
    double muh_mm1 = ld(g.c1h, m - 1) * mt + ld(g.c2h, m - 1);
    double dz = 2.0 / (ld(g.rdnw, m) + ld(g.rdnw, m - 1));
    double mu_face = 0.5 * (muh_m + muh_mm1);
    double cr = romv * a.dt / dz / mu_face;
    double ab = fabs(cr);
    lo = mu_face * (dz / a.dt) * (0.5 * dmin(1.0, cr + ab) * qo(m - 1, j, i) + 0.5 * dmax(-1.0, cr - ab) * qo(m, j, i));
    auto qc = [&](int kk) { return qf(kk, j, i); };
    double hi = vflux3_at(g, m, romv, qc);
    an = hi - lo;
  };
  xf(i, cf.lx0, cf.ax0);
  xf(i + 1, cf.lx1, cf.ax1);
  yf(j, cf.ly0, cf.ay0);
  yf(j + 1, cf.ly1, cf.ay1);
  zf(k, cf.lz0, cf.az0);
  zf(k + 1, cf.lz1, cf.az1);
}

template <typename QF, typename QO>
__device__ __forceinline__ void cell_scales(const Grid &g, const LimArgs &a, int k, int j, int i, QF qf, QO qo,
                                            double &s1, double &s2) {
  CellFluxes cf;
  cell_fluxes(g, a, k, j, i, qf, qo, cf);
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double msftx = ld(g.msftx, ix2(j, i, nx));
  const double rdzw = ld(g.rdnw, k);
  const double mass_old = ld(g.c1h, k) * ld(a.mu_old, ix2(j, i, nx)) + ld(g.c2h, k);
  const double fo = qo(k, j, i);
  const double div_low = msftx * msftx * (g.rdx * (cf.lx1 - cf.lx0) + g.rdy * (cf.ly1 - cf.ly0)) +
                         msftx * rdzw * (cf.lz1 - cf.lz0);
  const double ph_low = mass_old * fo - a.dt * div_low;
  auto pos = [](double x) { return dmax(0.0, x); };
  auto neg = [](double x) { return dmin(0.0, x); };
  const double flux_out = a.dt * (msftx * msftx * (g.rdx * (pos(cf.ax1) - neg(cf.ax0)) + g.rdy * (pos(cf.ay1) - neg(cf.ay0))) +
                                  msftx * rdzw * (neg(cf.az1) - pos(cf.az0)));
  if (a.opt == 1) {
    s1 = (flux_out > ph_low) ? dmax(0.0, ph_low / (flux_out + PD_EPS)) : 1.0;
    s2 = s1;
  } else {
    double qmax = fo, qmin = fo;
    const double nb[6] = {qo(k, j, i - 1), qo(k, j, i + 1), qo(k, j - 1, i), qo(k, j + 1, i),
                          qo(k == 0 ? 0 : k - 1, j, i), qo(k == nz - 1 ? nz - 1 : k + 1, j, i)};
    // x then y (periodic), then z (clamped), as _neighbour_min_max.
    qmax = dmax(qmax, dmax(nb[0], nb[1]));
    qmin = dmin(qmin, dmin(nb[0], nb[1]));
    qmax = dmax(qmax, dmax(nb[2], nb[3]));
    qmin = dmin(qmin, dmin(nb[2], nb[3]));
    qmax = dmax(qmax, dmax(nb[4], nb[5]));
    qmin = dmin(qmin, dmin(nb[4], nb[5]));
    const double flux_in = -a.dt * (msftx * msftx * (g.rdx * (neg(cf.ax1) - pos(cf.ax0)) + g.rdy * (neg(cf.ay1) - pos(cf.ay0))) +
                                    msftx * rdzw * (pos(cf.az1) - neg(cf.az0)));
    const double ph_hi = qmax * mass_old - ph_low;
    const double ph_lo = ph_low - qmin * mass_old;
    s1 = (flux_in > ph_hi) ? dmax(0.0, ph_hi / (flux_in + PD_EPS)) : 1.0;   // scale_in
    s2 = (flux_out > ph_lo) ? dmax(0.0, ph_lo / (flux_out + PD_EPS)) : 1.0;  // scale_out
  }
}

__global__ void k_lim_scale(Grid g, LimArgs a, const double *field, const double *field_old, double *s1, double *s2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny;
  if (i >= nx || j >= ny) return;
  auto qf = [&](int kk, int jj, int ii2) { return ld(field, ix3(kk, wrp(jj, ny), wrp(ii2, nx), ny, nx)) - a.offset; };
  auto qo = [&](int kk, int jj, int ii2) { return ld(field_old, ix3(kk, wrp(jj, ny), wrp(ii2, nx), ny, nx)) - a.offset; };
  double a1, a2;
  cell_scales(g, a, k, j, i, qf, qo, a1, a2);
  const size_t c = ix3(k, j, i, ny, nx);
  s1[c] = a1;
  s2[c] = a2;
}

__global__ void k_lim_tend(Grid g, LimArgs a, const double *field, const double *field_old, const double *s1,
                           const double *s2, const double *base, const double *mu_total_stage, double *tend_out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  auto qf = [&](int kk, int jj, int ii2) { return ld(field, ix3(kk, wrp(jj, ny), wrp(ii2, nx), ny, nx)) - a.offset; };
  auto qo = [&](int kk, int jj, int ii2) { return ld(field_old, ix3(kk, wrp(jj, ny), wrp(ii2, nx), ny, nx)) - a.offset; };
  CellFluxes cf;
  cell_fluxes(g, a, k, j, i, qf, qo, cf);
  auto S1 = [&](int kk, int jj, int ii2) { return ld(s1, ix3(kk, wrp(jj, ny), wrp(ii2, nx), ny, nx)); };
  auto S2 = [&](int kk, int jj, int ii2) { return ld(s2, ix3(kk, wrp(jj, ny), wrp(ii2, nx), ny, nx)); };
  double fx0, fx1, fy0, fy1, fz0, fz1;
  if (a.opt == 1) {
    auto limh = [&](double A, double s_m1, double s_c) { return A > 0.0 ? s_m1 * A : (A < 0.0 ? s_c * A : A); };
    fx0 = limh(cf.ax0, S1(k, j, i - 1), S1(k, j, i));
    fx1 = limh(cf.ax1, S1(k, j, i), S1(k, j, i + 1));
    fy0 = limh(cf.ay0, S1(k, j - 1, i), S1(k, j, i));
    fy1 = limh(cf.ay1, S1(k, j, i), S1(k, j + 1, i));
    auto limz = [&](double A, double below, double above) { return A < 0.0 ? below * A : (A > 0.0 ? above * A : A); };
    const double sc = S1(k, j, i);
    fz0 = limz(cf.az0, k == 0 ? sc : S1(k - 1, j, i), sc);
    fz1 = limz(cf.az1, sc, k + 1 >= nz ? sc : S1(k + 1, j, i));
  } else {
    // s_in = S1, s_out = S2
    auto limh = [&](double A, double in_c, double out_c, double in_m1, double out_m1) {
      return A > 0.0 ? dmin(in_c, out_m1) * A : dmin(out_c, in_m1) * A;
    };
    fx0 = limh(cf.ax0, S1(k, j, i), S2(k, j, i), S1(k, j, i - 1), S2(k, j, i - 1));
    fx1 = limh(cf.ax1, S1(k, j, i + 1), S2(k, j, i + 1), S1(k, j, i), S2(k, j, i));
    fy0 = limh(cf.ay0, S1(k, j, i), S2(k, j, i), S1(k, j - 1, i), S2(k, j - 1, i));
    fy1 = limh(cf.ay1, S1(k, j + 1, i), S2(k, j + 1, i), S1(k, j, i), S2(k, j, i));
    auto limz = [&](double A, double in_above, double out_above, double in_below, double out_below) {
      return A < 0.0 ? dmin(in_above, out_below) * A : dmin(out_above, in_below) * A;
    };
    const int kb = (k == 0) ? 0 : k - 1;      // cell below face k (padded)
    const int ka = (k + 1 >= nz) ? nz - 1 : k + 1;  // cell above face k+1 (padded)
    fz0 = limz(cf.az0, S1(k, j, i), S2(k, j, i), S1(kb, j, i), S2(kb, j, i));
    fz1 = limz(cf.az1, S1(ka, j, i), S2(ka, j, i), S1(k, j, i), S2(k, j, i));
  }
  fx0 = fx0 + cf.lx0;
  fx1 = fx1 + cf.lx1;
  fy0 = fy0 + cf.ly0;
  fy1 = fy1 + cf.ly1;
  fz0 = fz0 + cf.lz0;
  fz1 = fz1 + cf.lz1;
  const double msftx = ld(g.msftx, ix2(j, i, nx));
  double tend = -msftx * g.rdx * (fx1 - fx0);
  tend = tend - msftx * g.rdy * (fy1 - fy0);
  tend = tend - ld(g.rdnw, k) * (fz1 - fz0);
  const size_t c = ix3(k, j, i, ny, nx);
  if (base != nullptr) {
    const double mass_h = ld(g.c1h, k) * ld(mu_total_stage, ix2(j, i, nx)) + ld(g.c2h, k);
    tend_out[c] = ld(base, c) * mass_h + tend;
  } else {
    tend_out[c] = tend;
  }
}

// ---------------------------------------------------------------------------
// w faces: advect_w_flux (flux_advection.py:1277-1329, 1410-1482), pg_buoy_w
// (core/advance_w.py:146-290), cos-Coriolis/curvature (operational_mode.py:
// 1793-1822), rhs_ph (core/rhs_ph.py:175-401, order 2), w_work/ph_work
// (small_step_prep.py:322-323), ph_1 + phb, acoustic ww init.
// ---------------------------------------------------------------------------
struct WFaceOut {
  double *rw_tend, *ph_tend, *cqw, *w_w, *ph_w, *pt1, *ww;
  double *phb0;  // (ny, nx): base geopotential at the surface face (ht = phb0 / g)
};

__global__ void k_wface(Grid g, StateR s, StateR ref, const double *ru, const double *rv, const double *rom,
                        const double *ww_stage, const double *qtot, const double *mub, const double *mut,
                        const double *muts0, const double *muu, const double *muv, const double *base_w,
                        int top_lid, int moist_cqw, int w_coriolis, WFaceOut o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;  // face 0..nz
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  const size_t cw = ix3(k, j, i, ny, nx);
  const size_t c2d = ix2(j, i, nx);
  // ---- w advection ----
  auto ruw = [&](int jj, int ii2) {
    if (k == 0) return ld(ru, ix3(0, jj, ii2, ny, nx));
    if (k == nz) return ld(ru, ix3(nz - 1, jj, ii2, ny, nx));
    return ld(g.fnm, k) * ld(ru, ix3(k, jj, ii2, ny, nx)) + ld(g.fnp, k) * ld(ru, ix3(k - 1, jj, ii2, ny, nx));
  };
  auto rvw = [&](int jj, int ii2) {
    if (k == 0) return ld(rv, ix3(0, jj, ii2, ny, nx));
    if (k == nz) return ld(rv, ix3(nz - 1, jj, ii2, ny, nx));
    return ld(g.fnm, k) * ld(rv, ix3(k, jj, ii2, ny, nx)) + ld(g.fnp, k) * ld(rv, ix3(k - 1, jj, ii2, ny, nx));
  };
  auto wq = [&](int kk, int jj, int ii2) { return ld(s.w, ix3(kk, wrp(jj, ny), wrp(ii2, nx), ny, nx)); };
  const double msftx = ld(g.msftx, c2d);
  auto fqx = [&](int m) {
    int rm = wrp(m, nx);
    double vel = ruw(j, rm);
    return vel * flux5(wq(k, j, rm - 3), wq(k, j, rm - 2), wq(k, j, rm - 1), wq(k, j, rm), wq(k, j, rm + 1),
                       wq(k, j, rm + 2), vel);
  };
  double adv = -msftx * g.rdx * (fqx(i + 1) - fqx(i));
  if (ny > 1) {
    auto fqy = [&](int n) {
      int rn = wrp(n, ny);
      double vel = rvw(rn, i);
      return vel * flux5(wq(k, rn - 3, i), wq(k, rn - 2, i), wq(k, rn - 1, i), wq(k, rn, i), wq(k, rn + 1, i),
                         wq(k, rn + 2, i), vel);
    };
    adv = adv - msftx * g.rdy * (fqy(j + 1) - fqy(j));
  }
  {
    auto wc = [&](int kk) { return ld(s.w, ix3(kk, j, i, ny, nx)); };
    auto velf = [&](int m) {  // 0.5*(rom(m)+rom(m-1)), m>=1
      return 0.5 * (ld(rom, ix3(m, j, i, ny, nx)) + ld(rom, ix3(m - 1, j, i, ny, nx)));
    };
    auto vfw = [&](int m) {
      if (m <= 0) return 0.0;
      if (m == 1) return velf(1) * 0.5 * (wc(1) + wc(0));
      if (m < nz) return flux3v(wc(m - 2), wc(m - 1), wc(m), wc(m + 1), velf(m));
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
  // ---- pg_buoy_w (stage grid%p = state p', mu' = mut - mub) ----
  const double mub_c = ld(mub, c2d), mut_c = ld(mut, c2d);
  const double mu_prime = mut_c - mub_c;
  const double minv = 1.0 / ld(g.msfty, c2d);
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
    auto lev = [&](int kk, double &ru_m, double &u_m, double &rv_m, double &v_m) {
      const double c1 = ld(g.c1h, kk), c2 = ld(g.c2h, kk);
      const double u0 = ld(s.u, ix3(kk, j, i, ny, nx + 1)), u1 = ld(s.u, ix3(kk, j, i + 1, ny, nx + 1));
      const double v0 = ld(s.v, ix3(kk, j, i, ny + 1, nx)), v1 = ld(s.v, ix3(kk, j + 1, i, ny + 1, nx));
      const double rs0 = (c1 * muu_i + c2) * u0 / fuy_i, rs1 = (c1 * muu_ip + c2) * u1 / fuy_ip;
      const double vs0 = (c1 * muv_j + c2) * v0 / fvx_j, vs1 = (c1 * muv_jp + c2) * v1 / fvx_jp;
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
    const double mxy = ld(g.msftx, c2d) / ld(g.msfty, c2d);
    const double cor = ld(g.e, c2d) * (ld(g.cosa, c2d) * ru_f - mxy * ld(g.sina, c2d) * rv_f);
    const double curv = W_RERADIUS * (ru_f * u_f + mxy * rv_f * v_f);
    rw = rw + (cor + curv);
  }
  o.rw_tend[cw] = rw;
  o.cqw[cw] = cqw;
  // ---- rhs_ph (order 2, periodic) ----
  {
    auto pht = [&](int kk, int jj, int ii2) {
      const size_t cc = ix3(kk, wrp(jj, ny), wrp(ii2, nx), ny, nx);
      const double p = ld(s.ph_pert, cc);
      return p + (ld(s.ph_total, cc) - p);
    };
    double out = 0.0;
    if (k >= 1 && k <= nz - 1) {
      auto wdwn = [&](int m) {  // mass level m
        const double wwm = 0.5 * (ld(ww_stage, ix3(m + 1, j, i, ny, nx)) + ld(ww_stage, ix3(m, j, i, ny, nx)));
        return wwm * ld(g.rdnw, m) * (pht(m + 1, j, i) - pht(m, j, i));
      };
      const double term3 = ld(g.fnm, k) * wdwn(k) + ld(g.fnp, k) * wdwn(k - 1);
      out = 0.0 + (-term3);
      const double mass_f = ld(g.c1f, k) * mut_c + ld(g.c2f, k);
      out = out + mass_f * G * ld(s.w, cw) * minv;
      const double c1f = ld(g.c1f, k), c2f = ld(g.c2f, k);
      // y (v) advection
      auto vpair = [&](int jv) { return ld(s.v, ix3(k, jv, i, ny + 1, nx)) + ld(s.v, ix3(k - 1, jv, i, ny + 1, nx)); };
      auto muvf = [&](int jv) { return c1f * ld(muv, ix2(jv, i, nx)) + c2f; };
      const double pti = pht(k, j, i);
      const double dn_ = pht(k, j + 1, i) - pti;
      const double ds_ = pti - pht(k, j - 1, i);
      const double flux_y = muvf(j + 1) * vpair(j + 1) * dn_ + muvf(j) * vpair(j) * ds_;
      out = out + (-(0.25 * g.rdy * minv)) * flux_y;
      auto upair = [&](int iu) { return ld(s.u, ix3(k, j, iu, ny, nx + 1)) + ld(s.u, ix3(k - 1, j, iu, ny, nx + 1)); };
      auto muuf = [&](int iu) { return c1f * ld(muu, ix2(j, iu, nx + 1)) + c2f; };
      const double de_ = pht(k, j, i + 1) - pti;
      const double dw_ = pti - pht(k, j, i - 1);
      const double flux_x = muuf(i + 1) * upair(i + 1) * de_ + muuf(i) * upair(i) * dw_;
      out = out + (-(0.25 * g.rdx * minv)) * flux_x;
    } else if (k == nz && !top_lid) {
      const double mass_f = ld(g.c1f, nz) * mut_c + ld(g.c2f, nz);
      out = mass_f * G * ld(s.w, cw) * minv;
    }
    o.ph_tend[cw] = out;
  }
  // ---- prep work arrays ----
  const double mass_f_ref = ld(g.c1f, k) * ld(muts0, c2d) + ld(g.c2f, k);
  const double mass_f_cur = ld(g.c1f, k) * mut_c + ld(g.c2f, k);
  o.w_w[cw] = (mass_f_ref * ld(ref.w, cw) - mass_f_cur * ld(s.w, cw)) / ld(g.msfty, c2d);
  const double php = ld(s.ph_pert, cw);
  o.ph_w[cw] = ld(ref.ph_pert, cw) - php;
  o.pt1[cw] = ld(ref.ph_pert, cw) + (ld(s.ph_total, cw) - php);
  o.ww[cw] = ld(ww_stage, cw);
  if (k == 0) o.phb0[c2d] = ld(s.ph_total, cw) - php;
}

// ---------------------------------------------------------------------------
// Column kernel: calc_coef_w (acoustic_wrf.py:783-852) and the step-0
// calc_p_rho (core/calc_p_rho.py:52-134); seeds p, pm1, al and t_2ave.
// ---------------------------------------------------------------------------
struct CoefOut {
  double *a, *alpha, *gamma, *p, *pm1, *al, *t2ave;
};

__global__ void k_coef(Grid g, const double *mut, const double *muts0, const double *mu_work0, const double *c2a,
                       const double *cqw, const double *alt, const double *theta_w, const double *ph_w,
                       const double *ref_theta, double cof, int top_lid, CoefOut o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  const size_t c2d = ix2(j, i, nx);
  const double mt = ld(mut, c2d);
  auto mh = [&](int k) { return ld(g.c1h, k) * mt + ld(g.c2h, k); };
  auto mf = [&](int k) { return ld(g.c1f, k) * mt + ld(g.c2f, k); };
  auto C2A = [&](int k) { return ld(c2a, ix3(k, j, i, ny, nx)); };
  auto CQW = [&](int k) { return ld(cqw, ix3(k, j, i, ny, nx)); };
  const double lid = top_lid ? 0.0 : 1.0;
  const double rdnw_t = ld(g.rdnw, nz - 1);
  const double a_top = -2.0 * cof * (rdnw_t * rdnw_t) * C2A(nz - 1) * lid / (mh(nz - 1) * mf(nz - 1));
  o.a[ix3(0, j, i, ny, nx)] = 0.0;
  o.alpha[ix3(0, j, i, ny, nx)] = 1.0;
  o.gamma[ix3(0, j, i, ny, nx)] = 0.0;
  double gam_prev = 0.0;
  for (int k = 1; k < nz; ++k) {
    double ak = 0.0;
    if (k >= 2) {
      ak = -CQW(k) * cof * ld(g.rdn, k) * ld(g.rdnw, k - 1) * C2A(k - 1) / (mh(k - 1) * mf(k - 1));
    }
    const double b = 1.0 + CQW(k) * cof * ld(g.rdn, k) *
                               (ld(g.rdnw, k) * C2A(k) / (mh(k) * mf(k)) + ld(g.rdnw, k - 1) * C2A(k - 1) / (mh(k - 1) * mf(k)));
    const double cc = -CQW(k) * cof * ld(g.rdn, k) * ld(g.rdnw, k) * C2A(k) / (mh(k) * mf(k + 1));
    const double al_k = 1.0 / (b - ak * gam_prev);
    const double ga_k = cc * al_k;
    const size_t f = ix3(k, j, i, ny, nx);
    o.a[f] = ak;
    o.alpha[f] = al_k;
    o.gamma[f] = ga_k;
    gam_prev = ga_k;
  }
  const double b_top = 1.0 + 2.0 * cof * (rdnw_t * rdnw_t) * C2A(nz - 1) / (mh(nz - 1) * mf(nz));
  const size_t ft = ix3(nz, j, i, ny, nx);
  o.a[ft] = a_top;
  o.alpha[ft] = 1.0 / (b_top - a_top * gam_prev);
  o.gamma[ft] = 0.0;
  // step-0 calc_p_rho with muts = prep.muts and theta_1 = reference theta'
  const double muts = ld(muts0, c2d), mu_work = ld(mu_work0, c2d);
  for (int k = 0; k < nz; ++k) {
    const size_t c = ix3(k, j, i, ny, nx);
    const double mass_h = ld(g.c1h, k) * muts + ld(g.c2h, k);
    const double safe = safe12(mass_h);
    const double mu_term = ld(g.c1h, k) * mu_work;
    const double altc = ld(alt, c);
    const double al = -(altc * mu_term + ld(g.rdnw, k) * (ld(ph_w, ix3(k + 1, j, i, ny, nx)) - ld(ph_w, c))) / safe;
    const double t1 = ld(ref_theta, c) - T0;
    const double ttr = T0 + t1;
    const double sttr = fabs(ttr) > 1.0e-6 ? ttr : 1.0e-6;
    const double p = C2A(k) * (altc * (ld(theta_w, c) - mu_term * t1) / (safe * sttr) - al);
    o.p[c] = p;
    o.pm1[c] = p;
    o.al[c] = al;
    o.t2ave[c] = 0.0;
  }
}

}  // namespace wg
