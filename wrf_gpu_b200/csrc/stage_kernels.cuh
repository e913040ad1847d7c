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

// 16 resident blocks of 128 per SM (32 registers): timed at 433 x 433 x 50,
// 0.696 vs 0.735 ms/step with the compiler's 56 registers (12: 0.721).
#ifndef WG_DIAG_MINB
#define WG_DIAG_MINB 16
#endif
#if WG_DIAG_MINB > 0
#define WG_DIAG_BOUNDS __launch_bounds__(128, WG_DIAG_MINB)
#else
#define WG_DIAG_BOUNDS
#endif
__global__ void WG_DIAG_BOUNDS k_diag(Grid g, StateR s, int hyps, Diag o) {
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
template <typename F = double, typename Q>
__device__ __forceinline__ double vflux3_at(const Grid &g, int m, double romq, Q q) {
  const int nz = g.nz;
  if (m <= 0 || m >= nz) return 0.0;
  if (m == 1) return romq * (ld(g.fnm, 1) * q(1) + ld(g.fnp, 1) * q(0));
  if (m == nz - 1) return romq * (ld(g.fnm, nz - 1) * q(nz - 1) + ld(g.fnp, nz - 1) * q(nz - 2));
  return vflux3<F>(romq, q(m - 2), q(m - 1), q(m), q(m + 1));
}

// ---------------------------------------------------------------------------
// Outputs of the u-face stage kernel (tiled_faces.cuh):
// advect_u_flux (flux_advection.py:1131-1202) + base tendency,
// large-step PGF (rk_addtend_dry.py:303-317, 344-346), Coriolis
// (rk_addtend_dry.py:405-446), small_step_prep u_work (small_step_prep.py:319).
// ---------------------------------------------------------------------------
struct UFaceOut {
  double *u_tend, *u_w, *cqu;
};

// ---------------------------------------------------------------------------
// Outputs of the v-face stage kernel (tiled_faces.cuh):
// advect_v_flux (flux_advection.py:1205-1274) + base, PGF
// (rk_addtend_dry.py:320-341, 344-346), Coriolis (:448-466), v_work
// (small_step_prep.py:320).
// ---------------------------------------------------------------------------
struct VFaceOut {
  double *v_tend, *v_w, *cqv;
};

// Outputs of the mass-point stage kernel (tiled_stencils.cuh): theta and
// moisture tendencies (plain path), theta_work (small_step_prep.py:321).
struct MassOut {
  double *t_tend, *theta_w;
  double *q_tend[6];
  float *q_tend32[6];  // the mixed variant's float32 species tendencies
};
template <typename F>
struct MassOutQ;
template <>
struct MassOutQ<double> {
  __device__ static double *const (&get(const MassOut &o))[6] { return o.q_tend; }
};
template <>
struct MassOutQ<float> {
  __device__ static float *const (&get(const MassOut &o))[6] { return o.q_tend32; }
};

// ---------------------------------------------------------------------------
// Arguments of the positive-definite / monotonic limited scalar advection
// (flux_advection.py:736-1000; kernels in tiled_stencils.cuh).  Two passes:
// the scale pass writes the per-cell limiter scale(s), the tendency pass the
// limited tendency.
// ---------------------------------------------------------------------------
struct LimArgs {
  const double *ru, *rv, *rom;
  const double *mut;     // current total dry mass (ny, nx)
  const double *mu_old;  // start-of-step total dry mass (ny, nx)
  double dt;
  int opt;               // 1 PD, 2 mono
  double offset;         // subtracted from both fields (300 for theta, 0 for q)
  int deg;               // specified-boundary advection degradation (tiered faces, masked divergence)
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

// ---------------------------------------------------------------------------
// Outputs of the w-face stage kernel (tiled_faces.cuh):
// advect_w_flux (flux_advection.py:1277-1329, 1410-1482), pg_buoy_w
// (core/advance_w.py:146-290), cos-Coriolis/curvature (operational_mode.py:
// 1793-1822), rhs_ph (core/rhs_ph.py:175-401, order 2), w_work/ph_work
// (small_step_prep.py:322-323), ph_1 + phb, acoustic ww init.
// ---------------------------------------------------------------------------
struct WFaceOut {
  double *rw_tend, *ph_tend, *cqw, *w_w, *ph_w, *pt1, *ww;
  double *phb0;  // (ny, nx): base geopotential at the surface face (ht = phb0 / g)
};

// ---------------------------------------------------------------------------
// calc_coef_w (acoustic_wrf.py:783-852) and the step-0 calc_p_rho
// (core/calc_p_rho.py:52-134), which seeds p, pm1, al and t_2ave.
// A block owns 32 adjacent columns of one row j; its COEF_TY level lanes form
// the tridiagonal rows (a, b, c of every level) and the step-0 calc_p_rho
// level-parallel, and only the factorisation alpha(k) = 1 / (b - a*gamma(k-1)),
// gamma(k) = c * alpha(k) runs serially, one thread per column, out of shared
// memory.  Operation order is the reference's.
// ---------------------------------------------------------------------------
struct CoefOut {
  double *a, *alpha, *gamma, *p, *pm1, *al, *t2ave;
};

constexpr int COEF_TY = 8;
inline size_t coef_smem_bytes(int nz) { return (size_t)3 * (nz + 1) * 32 * sizeof(double); }

#ifdef WG_COEF_MINB
#define WG_COEF_BOUNDS __launch_bounds__(32 * COEF_TY, WG_COEF_MINB)
#else
#define WG_COEF_BOUNDS __launch_bounds__(32 * COEF_TY)
#endif
__global__ void WG_COEF_BOUNDS k_coef(Grid g, const double *mut, const double *muts0,
                                                       const double *mu_work0, const double *c2a, const double *cqw,
                                                       const double *alt, const double *theta_w, const double *ph_w,
                                                       const double *ref_theta, double cof, int top_lid, CoefOut o) {
  extern __shared__ double sm[];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz, L = nz + 1;
  const int i = blockIdx.x * 32 + tx, j = blockIdx.y;
  const bool valid = i < nx;
  // rows: SA = sub-diagonal a, SB = diagonal b -> alpha, SC = super-diagonal c -> gamma
  auto SA = [&](int k) -> double & { return sm[(size_t)k * 32 + tx]; };
  auto SB = [&](int k) -> double & { return sm[(size_t)(L + k) * 32 + tx]; };
  auto SC = [&](int k) -> double & { return sm[(size_t)(2 * L + k) * 32 + tx]; };
  auto M = [&](int k) { return ix3(k, j, i, ny, nx); };
  if (valid) {
    const size_t c2d = ix2(j, i, nx);
    const double mt = ld(mut, c2d);
    auto mh = [&](int k) { return ld(g.c1h, k) * mt + ld(g.c2h, k); };
    auto mf = [&](int k) { return ld(g.c1f, k) * mt + ld(g.c2f, k); };
    auto C2A = [&](int k) { return ld(c2a, M(k)); };
    for (int k = 1 + ty; k < nz; k += COEF_TY) {
      const double cq = ld(cqw, M(k));
      double ak = 0.0;
      if (k >= 2) {
        ak = -cq * cof * ld(g.rdn, k) * ld(g.rdnw, k - 1) * C2A(k - 1) / (mh(k - 1) * mf(k - 1));
      }
      const double b = 1.0 + cq * cof * ld(g.rdn, k) *
                                 (ld(g.rdnw, k) * C2A(k) / (mh(k) * mf(k)) + ld(g.rdnw, k - 1) * C2A(k - 1) / (mh(k - 1) * mf(k)));
      const double cc = -cq * cof * ld(g.rdn, k) * ld(g.rdnw, k) * C2A(k) / (mh(k) * mf(k + 1));
      SA(k) = ak;
      SB(k) = b;
      SC(k) = cc;
    }
    if (ty == COEF_TY - 1) {  // top row: a and b of face nz
      const double lid = top_lid ? 0.0 : 1.0;
      const double rdnw_t = ld(g.rdnw, nz - 1);
      SA(nz) = -2.0 * cof * (rdnw_t * rdnw_t) * C2A(nz - 1) * lid / (mh(nz - 1) * mf(nz - 1));
      SB(nz) = 1.0 + 2.0 * cof * (rdnw_t * rdnw_t) * C2A(nz - 1) / (mh(nz - 1) * mf(nz));
    }
    // step-0 calc_p_rho with muts = prep.muts and theta_1 = reference theta'
    const double muts = ld(muts0, c2d), mu_work = ld(mu_work0, c2d);
    for (int k = ty; k < nz; k += COEF_TY) {
      const size_t c = M(k);
      const double mass_h = ld(g.c1h, k) * muts + ld(g.c2h, k);
      const double safe = safe12(mass_h);
      const double mu_term = ld(g.c1h, k) * mu_work;
      const double altc = ld(alt, c);
      const double al = -(altc * mu_term + ld(g.rdnw, k) * (ld(ph_w, M(k + 1)) - ld(ph_w, c))) / safe;
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
  __syncthreads();
  if (ty == 0 && valid) {
    constexpr int SU = 8;  // levels per batch of shared-memory loads ahead of the chain
    double gam_prev = 0.0;
    int k = 1;
    for (; k + SU <= nz; k += SU) {
      double ra[SU], rb[SU], rc[SU];
#pragma unroll
      for (int u = 0; u < SU; ++u) {
        ra[u] = SA(k + u);
        rb[u] = SB(k + u);
        rc[u] = SC(k + u);
      }
#pragma unroll
      for (int u = 0; u < SU; ++u) {
        const double al_k = 1.0 / (rb[u] - ra[u] * gam_prev);
        const double ga_k = rc[u] * al_k;
        SB(k + u) = al_k;
        SC(k + u) = ga_k;
        gam_prev = ga_k;
      }
    }
    for (; k < nz; ++k) {
      const double al_k = 1.0 / (SB(k) - SA(k) * gam_prev);
      const double ga_k = SC(k) * al_k;
      SB(k) = al_k;
      SC(k) = ga_k;
      gam_prev = ga_k;
    }
    SB(nz) = 1.0 / (SB(nz) - SA(nz) * gam_prev);
    SC(nz) = 0.0;
    SA(0) = 0.0;
    SB(0) = 1.0;
    SC(0) = 0.0;
  }
  __syncthreads();
  if (valid) {
    for (int f = ty; f <= nz; f += COEF_TY) {
      const size_t c = M(f);
      o.a[c] = SA(f);
      o.alpha[c] = SB(f);
      o.gamma[c] = SC(f);
    }
  }
}

}  // namespace wg
