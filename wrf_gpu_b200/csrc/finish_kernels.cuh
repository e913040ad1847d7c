// End-of-stage kernels: small_step_finish (core/small_step_finish.py:419-498),
// the grid%p refresh (runtime/operational_mode.py:2169-2231 ->
// dynamics/acoustic_wrf.py:322-438), the large-step moisture update
// (operational_mode.py:3270-3316) and the carry outputs
// (operational_mode.py:2234-2265).
#pragma once
#include "dycore_common.cuh"

namespace wg {

__device__ __forceinline__ double safe_den(double x) {
  return fabs(x) > 1.0e-12 ? x : (x >= 0.0 ? 1.0e-12 : -1.0e-12);
}

__global__ void k_finish_u(Grid g, const double *u_w, const double *u_save, const double *muu, const double *muus,
                           double *u_out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny;
  if (i > nx || j >= ny) return;
  const size_t cu = ix3(k, j, i, ny, nx + 1);
  const size_t f2 = ix2(j, i, nx + 1);
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  const double ms = c1 * ld(muus, f2) + c2;
  const double mc = c1 * ld(muu, f2) + c2;
  u_out[cu] = (ld(g.msfuy, f2) * ld(u_w, cu) + ld(u_save, cu) * mc) / safe_den(ms);
}

__global__ void k_finish_v(Grid g, const double *v_w, const double *v_save, const double *muv, const double *muvs,
                           double *v_out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny;
  if (i >= nx || j > ny) return;
  const size_t cv = ix3(k, j, i, ny + 1, nx);
  const size_t f2 = ix2(j, i, nx);
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  const double ms = c1 * ld(muvs, f2) + c2;
  const double mc = c1 * ld(muv, f2) + c2;
  v_out[cv] = (ld(g.msfvx, f2) * ld(v_w, cv) + ld(v_save, cv) * mc) / safe_den(ms);
}

struct FinishArgs {
  // acoustic results
  const double *w_w, *ph_w, *theta_w, *p_ac, *mu_ac, *muts_ac, *t2ave, *ww_ac;
  const double *mut, *ww_stage;
  const double *q_tend[6];
  const float *q_tend32[6];  // the mixed variant's float32 species tendencies (q32)
  int q32;
  double dt_rk;
  int hyps, moist;
  // carry outputs (nullable: written on the final stage only)
  double *t_2ave_out, *ww_out, *t_save_out;
};

// One thread per (k, j, i) with k in 0..nz: face work (w, ph, ww) for every
// k, mass work (theta, p refresh, moisture, t_2ave, t_save) for k < nz and
// the 2-D mass fields at k == 0.  The refresh recomputes the finished ph' at
// k and k+1 from its inputs, with the same arithmetic as the face work.
// 12 resident blocks of 128 per SM (40 registers): timed at 433 x 433 x 50,
// 1.44 vs 1.61 ms/step with the compiler's 62 registers (10: 1.51, 14 / 16:
// 1.60).
#ifndef WG_FINISH_MINB
#define WG_FINISH_MINB 12
#endif
#if WG_FINISH_MINB > 0
#define WG_FINISH_BOUNDS __launch_bounds__(128, WG_FINISH_MINB)
#else
#define WG_FINISH_BOUNDS
#endif
__global__ void WG_FINISH_BOUNDS k_finish_cells(Grid g, StateR s, StateR origin, FinishArgs a, StateW o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  const size_t c2d = ix2(j, i, nx);
  auto M = [&](int kk) { return ix3(kk, j, i, ny, nx); };
  const double muts = ld(a.muts_ac, c2d);
  const double mut = ld(a.mut, c2d);
  const double mu_ac = ld(a.mu_ac, c2d);
  const double mu_base = ld(s.mu_total, c2d) - ld(s.mu_pert, c2d);
  const double mu_total_out = mu_base + mu_ac;
  auto ph_out = [&](int f, double &php, double &pht) {
    php = ld(a.ph_w, M(f)) + ld(s.ph_pert, M(f));
    const double phb = ld(s.ph_total, M(f)) - ld(s.ph_pert, M(f));
    pht = phb + php;
  };
  {
    const int f = k;
    const double msfty = ld(g.msfty, c2d);
    const double ms = ld(g.c1f, f) * muts + ld(g.c2f, f);
    const double mc = ld(g.c1f, f) * mut + ld(g.c2f, f);
    o.w[M(f)] = (msfty * ld(a.w_w, M(f)) + ld(s.w, M(f)) * mc) / safe_den(ms);
    double php, pht;
    ph_out(f, php, pht);
    o.ph_pert[M(f)] = php;
    o.ph_total[M(f)] = pht;
    if (a.ww_out != nullptr) a.ww_out[M(f)] = ld(a.ww_ac, M(f)) + ld(a.ww_stage, M(f));
  }
  if (k == 0) {
    o.mu_total[c2d] = mu_total_out;
    o.mu_pert[c2d] = mu_ac;
  }
  if (k >= nz) return;
  const double mub = mu_base;
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  const double ms = c1 * muts + c2;
  const double mc = c1 * mut + c2;
  const double t_save = ld(s.theta, M(k)) - T0;
  const double theta_out = (ld(a.theta_w, M(k)) + t_save * mc) / safe_den(ms) + T0;
  o.theta[M(k)] = theta_out;
  const double p_base = ld(s.p_total, M(k)) - ld(s.p_pert, M(k));
  const double pac = ld(a.p_ac, M(k));
  const double p_total1 = p_base + pac;
  double php0, pht0, php1, pht1;
  ph_out(k, php0, pht0);
  ph_out(k + 1, php1, pht1);
  const double phb0 = pht0 - php0, phb1 = pht1 - php1;
  double al, alb_used;
  if (a.hyps == 2) {
    const double muts_r = mub + mu_ac;
    const double c3f0 = ld(g.c3f, k), c3f1 = ld(g.c3f, k + 1), c4f0 = ld(g.c4f, k), c4f1 = ld(g.c4f, k + 1);
    const double c3h = ld(g.c3h, k), c4h = ld(g.c4h, k);
    double pfu = c3f1 * mub + c4f1 + g.p_top, pfd = c3f0 * mub + c4f0 + g.p_top, phm = c3h * mub + c4h + g.p_top;
    alb_used = (phb1 - phb0) / phm / log(pfd / pfu);
    const double dph_tot = (phb1 + php1) - (phb0 + php0);
    pfu = c3f1 * muts_r + c4f1 + g.p_top;
    pfd = c3f0 * muts_r + c4f0 + g.p_top;
    phm = c3h * muts_r + c4h + g.p_top;
    al = dph_tot / phm / log(pfd / pfu) - alb_used;
  } else {
    const double mhb = c1 * mub + c2;
    const double den = ld(g.dnw, k) * mhb;
    const double alb = -(phb1 - phb0) / (fabs(den) > 1.0e-12 ? den : 1.0e-12);
    const double muts_r = mub + mu_ac;
    const double mw = c1 * muts_r + c2;
    al = -(alb * c1 * mu_ac + ld(g.rdnw, k) * (php1 - php0)) / safe12(mw);
    alb_used = alb;
  }
  const double alt = al + alb_used;
  const double p_pert2 = pressure_from_theta_alt(theta_out, alt) - p_base;
  o.p_total[M(k)] = (p_total1 - pac) + p_pert2;
  o.p_pert[M(k)] = p_pert2;
  if (a.moist) {
    const double mass_old = c1 * ld(origin.mu_total, c2d) + c2;
    const double mass_new = c1 * mu_total_out + c2;
    const double inv = 1.0 / mass_new;
    for (int sp = 0; sp < 6; ++sp) {
      const double qt = a.q32 ? ld(a.q_tend32[sp], M(k)) : ld(a.q_tend[sp], M(k));
      o.q[sp][M(k)] = (mass_old * ld(origin.q[sp], M(k)) + a.dt_rk * qt) * inv;
    }
  } else if (o.q[0] != nullptr && s.q[0] != nullptr) {
    for (int sp = 0; sp < 6; ++sp) o.q[sp][M(k)] = ld(s.q[sp], M(k));
  }
  if (a.t_2ave_out != nullptr) a.t_2ave_out[M(k)] = ld(a.t2ave, M(k)) + T0;
  if (a.t_save_out != nullptr) a.t_save_out[M(k)] = t_save + T0;
}

}  // namespace wg
