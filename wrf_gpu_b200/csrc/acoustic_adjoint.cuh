// Vector-Jacobian product of one acoustic small step (advance_uv,
// advance_mu_t, advance_w, calc_p_rho with smdiv memory; the reference's
// acoustic_substep_core, core/acoustic.py:837-1150) with respect to its
// evolving work state, the stage constants held fixed.  Doubly periodic or
// specified domains (the frozen ring, the drain limiter with its scale held
// at the forward value, the relax-zone blend), no w_damping CFL term.
//
// The step is affine in the work state except through the new muts, which
// enters the denominators of t_2ave, of the ph update and of calc_p_rho; the
// reverse pass therefore needs the forward output X' = F(X), which the host
// computes first with the forward kernels.  Three kernels then run the
// reverse sweep:
//   * k_adj_column -- one thread per column, levels in reverse order of the
//                     forward phases: calc_p_rho + smdiv, the ph finish, the
//                     Thomas back and forward sweeps, the explicit w, the ph
//                     predictor, the omega-weighted theta / ph fluxes, t_2ave,
//                     the theta update, the mass update and the ww prefix.
//                     Leaves the cotangents of the horizontal theta flux
//                     divergence and of dvdxi per cell for:
//   * k_adj_faces  -- the u / v face cotangents gathered from the two cells
//                     each face bounds (the transpose of k_div_h), plus the
//                     outputs' own;
//   * k_adj_uv_faces, k_adj_uv_cells -- the transpose of advance_uv: every
//                     face forms its pressure-gradient weights, then every
//                     column gathers its four faces' shares into p, ph, al,
//                     muts and mudf in a fixed order (edge-clamped pairs
//                     alias), so the cotangents are the same on every run.
#pragma once
#include "dycore_common.cuh"
#include "acoustic_kernels.cuh"

namespace wg {

struct AcWork {
  double *u, *v, *w, *ph, *theta_w, *t2ave, *p, *pm1, *al, *ww, *mu, *muts, *muave, *mudf;
};
struct AcWorkR {
  const double *u, *v, *w, *ph, *theta_w, *t2ave, *p, *pm1, *al, *ww, *mu, *muts, *muave, *mudf;
};

struct AdjScratch {
  // mass-level: theta_w' bar (calc_p_rho part), theta flux divergence bar and
  // dvdxi bar; face-level: rhs bar (ph finish part), w bar, ww bar
  double *gthw, *gtend, *gdv, *grhs, *gws, *gww;
  double *fu[3], *fv[3];  // advance_uv transpose: per-face A1, B, mudf weight
};

// Cotangents of the stage tendencies (each nullable).
struct AdjTend {
  double *u_tend, *v_tend, *t_tend, *rw_tend, *ph_tend, *mu_tend;
};

struct AdjColArgs {
  AdjTend tc;             // tendency cotangents out
  const double *x0_muts;  // input muts (the drain limiter's mu_work_old)
  const double *dvdxi;    // forward dvdxi (specified: the drain limiter's dmdt)
  const double *mu_tend;  // nullable
  int specified;
  AcWorkR x1;  // forward output X' = F(X)
  AcWorkR co;  // cotangent of X'
  AcWork ci;   // cotangent of X (written)
  AdjScratch s;
  const double *alt, *c2a, *cqw, *theta_s, *pt1, *a, *alpha, *gamma, *mut;
  ColArgs col;  // dts, epssm, top_lid, damp_opt, dampcoef, zdamp, rzdamp
};

// One thread per column (i, j), three passes over the levels:
//   1 (up)   calc_p_rho + smdiv, the ph finish, the Thomas back substitution;
//   2 (down) the Thomas forward elimination, the explicit w, the ph predictor
//            one face behind it, the omega-weighted wd, t_2ave and theta;
//   3        the mass update, the ww prefix and the column sum of dvdxi.
// Pass 2 keeps the cotangents still collecting contributions (rhs, ph and w
// of faces m+1 and m, the buoyancy of level m, wd of level m+1) in registers
// and finishes each as soon as its last contributor has run.
// 6 resident 128-thread blocks per SM requested (85 registers): timed at
// 433 x 433 x 50, 1.96 vs 2.34 ms per VJP without the request (127 registers).
#ifndef WG_ADJCOL_MINB
#define WG_ADJCOL_MINB 6
#endif
#define WG_ADJCOL_BOUNDS __launch_bounds__(128, WG_ADJCOL_MINB)
__global__ void WG_ADJCOL_BOUNDS k_adj_column(Grid g, AdjColArgs q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  const size_t c2d = ix2(j, i, nx);
  const size_t plane = (size_t)ny * nx;
  const size_t base = (size_t)j * nx + i;
  auto M = [&](int k) { return (size_t)k * plane + base; };
  const double dts = q.col.dts, eps_p = 1.0 + q.col.epssm, eps_m = 1.0 - q.col.epssm;
  const double msfty = ld(g.msfty, c2d), minv = ld(g.rmsfty, c2d);
  const double mut = ld(q.mut, c2d), muts = ld(q.x1.muts, c2d);
  // specified domains advance mass, omega and theta on the interior columns only
  const bool active = !q.specified || (j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2);
  auto T1 = [&](int k) { return ld(q.theta_s, M(k)) - T0; };
  auto coef = [&](int k) {  // advance_w's stage-constant c2a*rdnw/mass_h(mut)
    return ld(q.c2a, M(k)) * ld(g.rdnw, k) / safe12(ld(g.c1h, k) * mut + ld(g.c2h, k));
  };
  double *__restrict__ s_thw = q.s.gthw;
  double *__restrict__ s_rhs = q.s.grhs;
  double *__restrict__ s_ws = q.s.gws;
  double *__restrict__ s_ww = q.s.gww;
  double *__restrict__ s_tend = q.s.gtend;
  double *__restrict__ s_dv = q.s.gdv;
  double g_muts = 0.0, g_muave = 0.0;

  // ================= pass 1 (faces f = 0..nz, level k = f) =================
  const double K = msfty * 0.5 * dts * G * eps_p;
  const bool do_damp = (q.col.damp_opt == 3 && q.col.dampcoef > 0.0);
  double dampmag = 0.0, hbot = 0.0;
  if (do_damp) {
    dampmag = dts * q.col.dampcoef;
    hbot = div_rcp(ld(q.pt1, M(nz)), G, RG) - q.col.zdamp;
  }
  double gal_prev = 0.0, gws_prev = 0.0, ph0 = 0.0;
  for (int f = 0; f <= nz; ++f) {
    // calc_p_rho with smdiv at level f: p' = pp + SMDIV (pp - pm1), pm1' = pp, al' = al
    double gal = 0.0;
    if (f < nz) {
      const size_t c = M(f);
      const double gp = ld(q.co.p, c);
      const double g_pp = (1.0 + SMDIV) * gp + ld(q.co.pm1, c);
      q.ci.pm1[c] = -SMDIV * gp;
      const double c2a = ld(q.c2a, c), alt = ld(q.alt, c);
      const double g_al = ld(q.co.al, c) - c2a * g_pp;
      const double c1 = ld(g.c1h, f);
      const double mass = c1 * muts + ld(g.c2h, f);
      const double safe = safe12(mass);
      const double t1 = T1(f);
      const double ttr = T0 + t1;
      const double sttr = fabs(ttr) > 1.0e-6 ? ttr : 1.0e-6;
      const double mu_term = c1 * (muts - mut);
      const double den = safe * sttr;
      // the sweep is serial per column: one reciprocal per divisor instead
      // of six divisions on its dependency chain
      const double rsafe = 1.0 / safe, rden = 1.0 / den;
      const double thw = ld(q.x1.theta_w, c), al = ld(q.x1.al, c);
      const double g_mu_term = -(c2a * alt * t1 * rden) * g_pp - (alt * rsafe) * g_al;
      const double g_safe = -(c2a * alt * (thw - mu_term * t1) * (rsafe * rden)) * g_pp - (al * rsafe) * g_al;
      g_muts += c1 * g_mu_term + (fabs(mass) > 1.0e-12 ? c1 * g_safe : 0.0);
      gal = ld(g.rdnw, f) * g_al * rsafe;  // al(f) = ... - rdnw (ph'(f+1) - ph'(f)) / safe
      s_thw[c] = ld(q.co.theta_w, c) + (c2a * alt * rden) * g_pp;
    }
    const size_t c = M(f);
    s_ww[c] = ld(q.co.ww, c);
    if (f == 0) {
      ph0 = ld(q.co.ph, c) + gal;  // ph'(0) = ph(0)
    } else {
      // ph finish: ph'(f) = rhs(f) + K ws(f) / (c1f muts + c2f)
      const double g_phn = ld(q.co.ph, c) - gal_prev + gal;
      const double mfs = ld(g.c1f, f) * muts + ld(g.c2f, f);
      const double rmfs = 1.0 / mfs;
      s_rhs[c] = g_phn;
      double g_ws = ld(q.co.w, c) + (K * rmfs) * g_phn;
      g_muts += -(K * ld(q.x1.w, c) * ld(g.c1f, f) * (rmfs * rmfs)) * g_phn;
      if (do_damp) {  // ws_out = (ws - dampwt mf w_save) / (1 + dampwt)
        const double hk = div_rcp(ld(q.pt1, c), G, RG);
        const double sv = sin(over_zdamp(0.5 * 3.141592653589793 * (hk - hbot), q.col));
        const double dampwt = (hk >= hbot) ? dampmag * (sv * sv) : 0.0;
        g_ws = g_ws / (1.0 + dampwt);
      }
      // Thomas back substitution ws(f-1) = wf(f-1) - gamma(f-1) ws(f), reversed
      if (f >= 2) g_ws = g_ws - ld(q.gamma, M(f - 1)) * gws_prev;
      s_ws[c] = g_ws;
      gws_prev = g_ws;
    }
    gal_prev = gal;
  }

  // ================= pass 2 (faces m = nz..1) =================
  const double c05dg = 0.5 * dts * G;
  const double wfac = dts * (0.5 * G * eps_m);
  // the ph predictor of face f: rhs(f) = ph(f) + msfty r / mf, r = dts (ph_tend + 0.5 g eps_m w)
  // - dts (fnm wd(f) + fnp wd(f-1)); returns the wd(f) (fnm) and wd(f-1) (fnp) cotangent parts
  auto predictor = [&](int f, double grhs, double &gph, double &gw, double &gwd_f, double &gwd_fm1) {
    if (f == nz && q.col.top_lid) grhs = 0.0;  // a rigid lid's rhs(nz) is zero
    gph += grhs;
    const double S = msfty * grhs / (ld(g.c1f, f) * mut + ld(g.c2f, f));
    gw += S * wfac;
    if (q.tc.ph_tend != nullptr) q.tc.ph_tend[M(f)] = dts * S;
    gwd_f = (f < nz) ? -(S * dts * ld(g.fnm, f)) : 0.0;
    gwd_fm1 = (f < nz) ? -(S * dts * ld(g.fnp, f)) : 0.0;
  };
  // wd(k) = 0.5 (ww'(k+1) + ww'(k)) rdnw (pt1(k+1) - pt1(k))
  auto wd_rev = [&](int k, double gwd) {
    const double cw = 0.5 * ld(g.rdnw, k) * (ld(q.pt1, M(k + 1)) - ld(q.pt1, M(k))) * gwd;
    s_ww[M(k + 1)] += cw;
    s_ww[M(k)] += cw;
  };
  // t_2ave' and theta at level k (after its buoyancy cotangent is complete)
  auto t2a_theta = [&](int k, double gbuoy, double gt2a_extra) {
    const size_t c = M(k);
    const double gt2a = ld(q.co.t2ave, c) + ld(q.c2a, c) * ld(q.alt, c) * gbuoy + gt2a_extra;
    const double c1 = ld(g.c1h, k);
    const double mass_h = c1 * muts + ld(g.c2h, k);
    const double t1 = T1(k);
    const double rd = 1.0 / (mass_h * (T0 + t1));
    const double gn = gt2a * rd;
    const double gthw = s_thw[c] + 0.5 * eps_p * gn;
    q.ci.t2ave[c] = 0.5 * eps_m * gn;
    g_muave += c1 * T0 * gn;
    g_muts += -(ld(q.x1.t2ave, c) * (T0 + t1) * rd) * c1 * gt2a;  // t2ave / mass_h
    // theta: thw' = thw + msfty dts t_tend - dts msfty (hdiv + rdnw (wdtn(k+1) - wdtn(k)))
    q.ci.theta_w[c] = gthw;
    const double gtend = active ? -dts * msfty * gthw : 0.0;  // a frozen column keeps its theta
    s_tend[c] = gtend;
    if (q.tc.t_tend != nullptr) q.tc.t_tend[c] = active ? msfty * dts * gthw : 0.0;
    if (!active) return;
    const double rdnw = ld(g.rdnw, k);
    if (k + 1 <= nz - 1) s_ww[M(k + 1)] += rdnw * gtend * (ld(g.fnm, k + 1) * T1(k + 1) + ld(g.fnp, k + 1) * t1);
    if (k >= 1) s_ww[c] -= rdnw * gtend * (ld(g.fnm, k) * t1 + ld(g.fnp, k) * T1(k - 1));
  };
  double gnext = 0.0;
  double R_hi = 0.0, R_mid = s_rhs[M(nz)];  // rhs cotangents of faces m+1, m
  double P_hi = 0.0, P_mid = 0.0;           // ph cotangents of faces m+1, m
  double W_hi = 0.0;                        // w cotangent of face m+1
  double B_mid = 0.0;                       // buoyancy cotangent of level m
  double D_hi = 0.0;                        // wd cotangent of level m+1 (from face m+2)
  double gt2a_top = 0.0;
  double coef_lo = 0.0;  // coef(m) of the next (lower) face, carried down
  for (int m = nz; m >= 1; --m) {
    const size_t c = M(m);
    // Thomas forward elimination wf(m) = (wn(m) - a(m) wf(m-1)) alpha(m), reversed
    const double gwf = s_ws[c] + gnext;
    const double alf = ld(q.alpha, c);
    const double gwn = alf * gwf;
    gnext = -ld(q.a, c) * alf * gwf;
    double R_lo = (m - 1 >= 1) ? s_rhs[M(m - 1)] : 0.0;
    double P_lo = (m - 1 == 0) ? ph0 : 0.0;
    double B_lo = 0.0;
    double W_mid = 0.0;
    if (q.tc.rw_tend != nullptr) q.tc.rw_tend[c] = (m <= nz - 1 || !q.col.top_lid) ? dts * gwn : 0.0;
    if (m <= nz - 1) {  // explicit w: wn = w + dts rw_tend + tA(rhs, ph) + tB(buoy, muave)
      W_mid = gwn;
      const double Q = minv * ld(q.cqw, c) * (c05dg * ld(g.rdn, m)) * gwn;
      const double cf = (m == nz - 1) ? coef(m) : coef_lo, cm = coef(m - 1);
      coef_lo = cm;
      R_hi += Q * cf * eps_p;
      R_mid -= Q * cf * eps_p + Q * cm * eps_p;
      R_lo += Q * cm * eps_p;
      P_hi += Q * cf * eps_m;
      P_mid -= Q * cf * eps_m + Q * cm * eps_m;
      P_lo += Q * cm * eps_m;
      const double R = dts * G * minv * gwn;
      B_mid += R * ld(g.rdn, m);
      B_lo -= R * ld(g.rdn, m);
      g_muave -= R * ld(g.c1f, m);
    } else if (!q.col.top_lid) {  // the open top face
      W_mid = gwn;
      const double gT = minv * gwn;
      const int km1 = nz - 1;
      const double mhm = safe12(ld(g.c1h, km1) * mut + ld(g.c2h, km1));
      const double rdnw_t = ld(g.rdnw, km1);
      const double CA = -0.5 * dts * G / mhm * (rdnw_t * rdnw_t) * 2.0 * ld(q.c2a, M(km1));
      R_mid += CA * eps_p * gT;
      R_lo -= CA * eps_p * gT;
      P_mid += CA * eps_m * gT;
      P_lo -= CA * eps_m * gT;
      gt2a_top = -dts * G * 2.0 * rdnw_t * ld(q.c2a, M(km1)) * ld(q.alt, M(km1)) * gT;
      g_muave += -dts * G * ld(g.c1f, nz) * gT;
    }
    if (m + 1 <= nz) {  // face m+1 has all its contributions
      double gwd_f, gwd_fm1;
      predictor(m + 1, R_hi, P_hi, W_hi, gwd_f, gwd_fm1);
      q.ci.ph[M(m + 1)] = P_hi;
      q.ci.w[M(m + 1)] = W_hi;
      if (m + 1 <= nz - 1) wd_rev(m + 1, D_hi + gwd_f);
      D_hi = gwd_fm1;
    }
    if (m <= nz - 1) t2a_theta(m, B_mid, (m == nz - 1) ? gt2a_top : 0.0);
    R_hi = R_mid; R_mid = R_lo;
    P_hi = P_mid; P_mid = P_lo;
    W_hi = W_mid;
    B_mid = B_lo;
  }
  {  // face 1, level 0 and face 0
    double gwd_f, gwd_fm1;
    predictor(1, R_hi, P_hi, W_hi, gwd_f, gwd_fm1);
    q.ci.ph[M(1)] = P_hi;
    q.ci.w[M(1)] = W_hi;
    if (1 <= nz - 1) wd_rev(1, D_hi + gwd_f);
    wd_rev(0, gwd_fm1);
    q.ci.ph[M(0)] = P_mid;
    q.ci.w[M(0)] = 0.0;  // the surface w is a stage constant
    if (q.tc.rw_tend != nullptr) q.tc.rw_tend[M(0)] = 0.0;
    if (q.tc.ph_tend != nullptr) q.tc.ph_tend[M(0)] = 0.0;
    t2a_theta(0, B_mid, (nz - 1 == 0) ? gt2a_top : 0.0);
  }

  // ================= pass 3: mass update, ww prefix, dvdxi sum =================
  const double gmu = ld(q.co.mu, c2d);
  const double g_muts_t = ld(q.co.muts, c2d) + g_muts;
  const double g_muave_t = ld(q.co.muave, c2d) + g_muave;
  if (!active) {  // mu, muts, muave, mudf and ww pass through unchanged
    q.ci.mu[c2d] = gmu;
    q.ci.muts[c2d] = g_muts_t;
    q.ci.muave[c2d] = g_muave_t;
    q.ci.mudf[c2d] = ld(q.co.mudf, c2d);
    for (int f = 0; f <= nz; ++f) q.ci.ww[M(f)] = s_ww[M(f)];
    for (int k = 0; k < nz; ++k) s_dv[M(k)] = 0.0;
    if (q.tc.mu_tend != nullptr) q.tc.mu_tend[c2d] = 0.0;
    return;
  }
  // the drain limiter's scale (dynamics/mu_t_advance.py:295-451), held fixed
  double scale = 1.0;
  if (q.specified) {
    double dmdt = 0.0;
    for (int k = 0; k < nz; ++k) {
      const double tk = ld(g.dnw, k) * ld(q.dvdxi, M(k));
      dmdt = (k == 0) ? tk : dmdt + tk;
    }
    const double mu_tend = (q.mu_tend != nullptr) ? ld(q.mu_tend, c2d) : 0.0;
    const double mu_work_old = ld(q.x0_muts, c2d) - mut;
    const double floor_ = dmax(MIN_MUTS_PA, MIN_MUTS_FRACTION * mut);
    const double muts_old = mut + mu_work_old;
    const double raw = dts * (dmdt + mu_tend);
    const double allowed = dmax(muts_old - floor_, 0.0);
    const double loss = -raw;
    const bool finite = isfinite(raw) && isfinite(muts_old);
    scale = (finite && (loss > allowed)) ? allowed / dmax(loss, 1.0) : (finite ? 1.0 : 0.0);
    scale = dmin(dmax(scale, 0.0), 1.0);
  }
  const double g_mwn = gmu + g_muts_t + 0.5 * eps_p * g_muave_t;  // mu_work' = mu_work + dts (dmdt + mu_tend)
  const double g_mwo = -gmu + 0.5 * eps_m * g_muave_t + g_mwn;
  q.ci.mu[c2d] = gmu;
  q.ci.muts[c2d] = g_mwo;
  q.ci.muave[c2d] = 0.0;
  double g_dmdt = dts * g_mwn + ld(q.co.mudf, c2d);
  // ww'(kk) = ww(0) - sum_{m <= kk} inc(m) - ww_1(kk), kk < nz; ww'(nz) = ww(nz)
  double S = 0.0;
  s_dv[M(nz - 1)] = 0.0;
  for (int m = nz - 1; m >= 1; --m) {
    S += s_ww[M(m)];
    const int k = m - 1;
    const double ginc = -S;
    g_dmdt += ld(g.dnw, k) * ld(g.c1h, k) * minv * ginc;
    s_dv[M(k)] = scale * (ld(g.dnw, k) * minv * ginc);
    q.ci.ww[M(m)] = 0.0;
  }
  q.ci.ww[M(0)] = S + s_ww[M(0)];
  q.ci.ww[M(nz)] = s_ww[M(nz)];
  // dmdt = sum_k dnw(k) dvdxi(k)
  g_dmdt = scale * g_dmdt;
  // mu_tend enters as dmdt does: (dmdt + mu_tend) scale and c1h dmdt + c1h mu_tend
  if (q.tc.mu_tend != nullptr) q.tc.mu_tend[c2d] = g_dmdt;
  for (int k = 0; k < nz; ++k) s_dv[M(k)] += ld(g.dnw, k) * g_dmdt;
}

struct AdjFaceArgs {
  const double *gtend, *gdv, *theta_s;
  const double *co_u, *co_v;
  double *ci_u, *ci_v;
  BdyArgs bdy;  // relax-zone weights (active on specified domains)
};

// The u / v face cotangents (after advance_uv): the outputs' own plus the
// transpose of the dvdxi and theta-flux divergence of the two cells a face
// bounds (k_div_h, doubly periodic).  Index space (nx+1) x (ny+1) x nz.
__global__ void k_adj_faces(Grid g, AdjFaceArgs q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nxu = nx + 1, nyv = ny + 1;
  if (i > nx || j > ny) return;
  auto T1 = [&](int jj, int ii) { return ld(q.theta_s, ix3(k, jj, ii, ny, nx)) - T0; };
  if (j < ny) {
    const size_t cu = ix3(k, j, i, ny, nxu);
    double gu = ld(q.co_u, cu);
    if (i >= 1) {  // east face of cell i-1
      const int cc = i - 1;
      const size_t c = ix3(k, j, cc, ny, nx), c2 = ix2(j, cc, nx);
      const double msftx = ld(g.msftx, c2), msfty = ld(g.msfty, c2);
      gu += msftx * msfty * g.rdx * ld(q.gdv, c) +
            msftx * (0.5 * g.rdx) * (T1(j, wrp(cc + 1, nx)) + T1(j, cc)) * ld(q.gtend, c);
    }
    if (i <= nx - 1) {  // west face of cell i
      const size_t c = ix3(k, j, i, ny, nx), c2 = ix2(j, i, nx);
      const double msftx = ld(g.msftx, c2), msfty = ld(g.msfty, c2);
      gu -= msftx * msfty * g.rdx * ld(q.gdv, c) +
            msftx * (0.5 * g.rdx) * (T1(j, i) + T1(j, wrp(i - 1, nx))) * ld(q.gtend, c);
    }
    // the relax-zone blend u' = u + wu (target - u)
    if (q.bdy.active) gu = gu - relax_weight_u(j, i, ny, nxu, q.bdy) * gu;
    q.ci_u[cu] = gu;
  }
  if (i < nx) {
    const size_t cv = ix3(k, j, i, nyv, nx);
    double gv = ld(q.co_v, cv);
    if (j >= 1) {  // north face of cell j-1
      const int cj = j - 1;
      const size_t c = ix3(k, cj, i, ny, nx), c2 = ix2(cj, i, nx);
      const double msftx = ld(g.msftx, c2), msfty = ld(g.msfty, c2);
      gv += msftx * msfty * g.rdy * ld(q.gdv, c) +
            msftx * (0.5 * g.rdy) * (T1(wrp(cj + 1, ny), i) + T1(cj, i)) * ld(q.gtend, c);
    }
    if (j <= ny - 1) {  // south face of cell j
      const size_t c = ix3(k, j, i, ny, nx), c2 = ix2(j, i, nx);
      const double msftx = ld(g.msftx, c2), msfty = ld(g.msfty, c2);
      gv -= msftx * msfty * g.rdy * ld(q.gdv, c) +
            msftx * (0.5 * g.rdy) * (T1(j, i) + T1(wrp(j - 1, ny), i)) * ld(q.gtend, c);
    }
    if (q.bdy.active) gv = gv - relax_weight_v(j, i, nyv, nx, q.bdy) * gv;
    q.ci_v[cv] = gv;
  }
}

struct AdjUVArgs {
  double *gu_tend, *gv_tend;  // u_tend / v_tend cotangents out (nullable)
  const double *gu, *gv;  // total cotangents of the advanced u, v
  const double *alt, *pb, *php, *cqu, *cqv, *muu, *muv;
  double *ci_p, *ci_ph, *ci_al, *ci_muts, *ci_mudf;  // accumulated (p, al, mudf from zero)
  double *fu[3], *fv[3];  // per-face A1, B and the mudf weight (u faces, v faces)
  double dts;
  int top_lid;
};

// Transpose of advance_uv's pressure-gradient and divergence-damping terms
// (the u / v work values themselves pass through with unit weight), in two
// passes so that every cotangent is summed in a fixed order: k_adj_uv_faces
// forms each face's three scalars -- A1 (the ph and p weight), B (the dpn
// weight) and the mudf weight -- and k_adj_uv_cells gathers them per cell.
// A face at position f of a row has the mass points a = max(f-1, 0) and
// C = min(f, n-1) (the edge faces' pairs alias), and in the forward update
// reads ph and p' through a difference C - a, al, pb and muts through a
// sum, and p' through the pair sums of dpn at up to three levels.
__global__ void k_adj_uv_faces(Grid g, AdjUVArgs q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nxu = nx + 1, nyv = ny + 1;
  if (i > nx || j > ny) return;
  const int ic = min(i, nx - 1), jc = min(j, ny - 1);
  const int oC = jc * nx + ic, oW = jc * nx + max(i - 1, 0), oS = max(j - 1, 0) * nx + ic;
  const size_t plane = (size_t)ny * nx;
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  auto face = [&](int oa, double gvel, double cq, double msfr, double mass, double rd, double md_coef, double *const *f,
                  size_t cf) {
    const double Gx = -q.dts * cq * gvel;
    f[0][cf] = msfr * 0.5 * rd * mass * Gx;
    f[1][cf] = msfr * rd * (ld(q.php, k * plane + oC) - ld(q.php, k * plane + oa)) * Gx;
    f[2][cf] = c1 * md_coef * gvel;
  };
  if (j < ny) {
    const int fu = j * nxu + i;
    const size_t cu = (size_t)k * ny * nxu + fu;
    const double msfr = div_msf(ld(g.msfux, fu), g.msfuy, g.rmsfuy, fu);
    face(oW, ld(q.gu, cu), ld(q.cqu, cu), msfr, c1 * ld(q.muu, fu) + c2, g.rdx, -EMDIV * g.dx * ld(g.rmsfuy, fu), q.fu,
         cu);
    if (q.gu_tend != nullptr) q.gu_tend[cu] = q.dts * ld(q.gu, cu);
  }
  if (i < nx) {
    const int fv = j * nx + i;
    const size_t cv = (size_t)k * nyv * nx + fv;
    const double msfr = div_msf(ld(g.msfvy, fv), g.msfvx, g.rmsfvx, fv);
    face(oS, ld(q.gv, cv), ld(q.cqv, cv), msfr, c1 * ld(q.muv, fv) + c2, g.rdy, -EMDIV * g.dy * ld(g.rmsfvx, fv), q.fv,
         cv);
    if (q.gv_tend != nullptr) q.gv_tend[cv] = q.dts * ld(q.gv, cv);
  }
}

// The geometry of a cell's four faces (u at i and i+1, v at j and j+1): their
// offsets and planes in the per-face arrays, the difference weights d =
// [cell is C] - [cell is a] and sum weights s = [cell is C] + [cell is a]
// (2 or 0 at an aliased edge face), and the other mass point of each pair.
struct CellFaces {
  size_t fo[4], fplane[4], other[4];
  double dw[4], sw[4];
  __device__ CellFaces(int i, int j, int nx, int ny) {
    const int nxu = nx + 1, nyv = ny + 1;
    fo[0] = (size_t)j * nxu + i; fo[1] = (size_t)j * nxu + i + 1;
    fo[2] = (size_t)j * nx + i; fo[3] = (size_t)(j + 1) * nx + i;
    fplane[0] = fplane[1] = (size_t)ny * nxu;
    fplane[2] = fplane[3] = (size_t)nyv * nx;
    other[0] = (size_t)j * nx + max(i - 1, 0); other[1] = (size_t)j * nx + min(i + 1, nx - 1);
    other[2] = (size_t)max(j - 1, 0) * nx + i; other[3] = (size_t)min(j + 1, ny - 1) * nx + i;
    dw[0] = i == 0 ? 0.0 : 1.0; dw[1] = i == nx - 1 ? 0.0 : -1.0;
    dw[2] = j == 0 ? 0.0 : 1.0; dw[3] = j == ny - 1 ? 0.0 : -1.0;
    sw[0] = i == 0 ? 2.0 : 1.0; sw[1] = i == nx - 1 ? 2.0 : 1.0;
    sw[2] = j == 0 ? 2.0 : 1.0; sw[3] = j == ny - 1 ? 2.0 : 1.0;
  }
  __device__ double F(const AdjUVArgs &q, int n, int comp, int k) const {
    const double *const *f = n < 2 ? q.fu : q.fv;
    return ld(f[comp], (size_t)k * fplane[n] + fo[n]);
  }
};

// One thread per cell (i, j, kk), kk = 0..nz: the cell's share of its four
// faces' A1 and B in ph, p and al, summed in a fixed order.
// 16 resident blocks of 128 per SM: the substep VJP 1.862 vs 1.878 ms at
// 433 x 433 x 50 unbounded (12: 1.905).
#ifndef WG_ADJCELL_MINB
#define WG_ADJCELL_MINB 16
#endif
#if WG_ADJCELL_MINB > 0
#define WG_ADJCELL_MINB_BOUNDS __launch_bounds__(128, WG_ADJCELL_MINB)
#else
#define WG_ADJCELL_MINB_BOUNDS
#endif
__global__ void WG_ADJCELL_MINB_BOUNDS k_adj_uv_cells(Grid g, AdjUVArgs q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int kk = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  const size_t plane = (size_t)ny * nx;
  const size_t c = (size_t)kk * plane + (size_t)j * nx + i;
  const CellFaces cf(i, j, nx, ny);
  // ph: face levels kk (its lower face) and kk - 1 (its upper face)
  double gph = 0.0;
  for (int k = kk - 1; k <= kk; ++k) {
    if (k < 0 || k >= nz) continue;
    for (int n = 0; n < 4; ++n) gph = gph + cf.dw[n] * cf.F(q, n, 0, k);
  }
  q.ci_ph[c] += gph;
  if (kk == nz) return;
  // sum-weighted B of the four faces at level k (the pair sums of dpn)
  auto Bs = [&](int k) {
    double b = 0.0;
    for (int n = 0; n < 4; ++n) b = b + cf.sw[n] * cf.F(q, n, 1, k);
    return b;
  };
  double gp = 0.0, gal = 0.0;
  const double alt_c = ld(q.alt, c), pb_c = ld(q.pb, c);
  for (int n = 0; n < 4; ++n) {
    const double A1 = cf.F(q, n, 0, kk);
    const size_t o = (size_t)kk * plane + cf.other[n];
    // p: + (alt_a + alt_C) A1 to C, - to a
    gp = gp + cf.dw[n] * ((ld(q.alt, o) + alt_c) * A1);
    // al: (pb_C - pb_a) A1 to both points (this cell is C of the W / S face
    // and a of the E / N face)
    const double pdiff = (n == 0 || n == 2) ? (pb_c - ld(q.pb, o)) : (ld(q.pb, o) - pb_c);
    gal = gal + cf.sw[n] * (pdiff * A1);
  }
  // dpn: the pair-sum weights reaching level kk from face levels kk - 1 .. kk + 1
  const double rd_k = ld(g.rdnw, kk);
  if (kk + 1 < nz) gp = gp + 0.5 * ld(g.fnp, kk + 1) * (rd_k * Bs(kk));
  if (kk >= 1) gp = gp + 0.5 * ld(g.fnm, kk) * (-rd_k * Bs(kk));
  else gp = gp + 0.5 * g.cf1 * (-rd_k * Bs(0));
  if (kk >= 1) gp = gp + 0.5 * ld(g.fnm, kk) * (ld(g.rdnw, kk - 1) * Bs(kk - 1));
  if (kk + 1 <= nz - 1) gp = gp + 0.5 * ld(g.fnp, kk + 1) * (-ld(g.rdnw, kk + 1) * Bs(kk + 1));
  if (kk == 1) gp = gp + 0.5 * g.cf2 * (-ld(g.rdnw, 0) * Bs(0));
  if (kk == 2) gp = gp + 0.5 * g.cf3 * (-ld(g.rdnw, 0) * Bs(0));
  if (q.top_lid) {
    const double rt = ld(g.rdnw, nz - 1);
    if (kk == nz - 1) gp = gp + 0.5 * g.cf1 * (rt * Bs(nz - 1));
    if (kk == nz - 2) gp = gp + 0.5 * g.cf2 * (rt * Bs(nz - 1));
    if (kk == nz - 3) gp = gp + 0.5 * g.cf3 * (rt * Bs(nz - 1));
  }
  q.ci_p[c] += gp;
  q.ci_al[c] += gal;
}

// One thread per column (i, j): the column sums of the four faces' muts and
// mudf shares, level by level.
__global__ void k_adj_uv_cols(Grid g, AdjUVArgs q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  const CellFaces cf(i, j, nx, ny);
  double muts = 0.0, mudf = 0.0;
  for (int k = 0; k < nz; ++k) {
    const double c1 = ld(g.c1h, k);
    for (int n = 0; n < 4; ++n) {
      muts = muts + cf.sw[n] * (-0.5 * c1 * cf.F(q, n, 1, k));
      mudf = mudf + cf.dw[n] * cf.F(q, n, 2, k);
    }
  }
  const size_t c2d = (size_t)j * nx + i;
  q.ci_muts[c2d] += muts;
  q.ci_mudf[c2d] += mudf;
}

}  // namespace wg
