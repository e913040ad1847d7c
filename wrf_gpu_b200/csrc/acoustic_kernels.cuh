// Acoustic substep kernels (fp64) and the end-of-stage finish.
//
// One substep is two launches:
//   k_advance_u / k_advance_v  -- advance_uv on every u / v face
//                                 (core/acoustic.py:626-786), face-parallel;
//   k_column                   -- advance_mu_t (dynamics/mu_t_advance.py),
//                                 advance_w with its Thomas solve
//                                 (core/advance_w.py:293-627) and calc_p_rho
//                                 with smdiv memory (core/calc_p_rho.py:137-183),
//                                 one thread per column.
// The column kernel writes only its own column and reads neighbours only of
// stage-constant arrays and of u/v (finished by the face kernels), so a
// substep has no intra-kernel race.
#pragma once
#include "dycore_common.cuh"

namespace wg {

// Acoustic work state (operational_mode.py:1996-2166 AcousticCoreState).
struct Acoustic {
  double *u, *v, *w, *ph, *theta_w, *t2ave, *p, *pm1, *al, *ww;  // evolving
  double *mu, *muts, *muave, *mudf;                              // evolving 2-D
  const double *u_tend, *v_tend, *t_tend, *rw_tend, *ph_tend;    // stage tendencies
  const double *alt, *pb, *c2a, *cqu, *cqv, *cqw, *php, *pt1;    // stage constants
  const double *a, *alpha, *gamma, *ww_1;
  const double *mut, *muu, *muv, *muus, *muvs;                   // stage 2-D
  const double *mu_tend;                                         // base mu tendency (nullable)
  const double *u_1, *v_1, *w_save;                              // stage u, v, w (u_save/v_save/w_save)
  const double *theta_s;                                         // stage theta (t_save = theta - 300)
  const double *phb0;                                            // stage base geopotential at face 0 (ny, nx)
};

struct BdyArgs {
  int active;
  const double *u_target, *v_target;  // work-array targets (u-face / v-face shapes)
  double sub_ratio;                   // strength * dts / dt_full
  int spec_zone, relax_zone;
};

// Weight of the per-substep convex blend toward the boundary work target
// (coupling/boundary_apply.py:803-855), DEFAULT_BOUNDARY_CONFIG widths.
__device__ __forceinline__ double relax_weight_u(int j, int i, int y_len, int x_len, const BdyArgs &b) {
  double w = 0.0;
  for (int d = 0; d < b.spec_zone; ++d) {
    if (i == d || i == x_len - 1 - d) w = 1.0;
  }
  for (int d = b.spec_zone; d < b.relax_zone; ++d) {
    double linear = (b.relax_zone > 1) ? dmax(0.0, (double)(b.spec_zone + b.relax_zone - (d + 1)) / (double)(b.relax_zone - 1)) : 0.0;
    double weight = dmin(1.0, dmax(0.0, b.sub_ratio * 0.1 * linear));
    if (j >= d + 1 && j < y_len - d - 1 && (i == d || i == x_len - 1 - d)) w = weight;
  }
  return w;
}

__device__ __forceinline__ double relax_weight_v(int j, int i, int y_len, int x_len, const BdyArgs &b) {
  double w = 0.0;
  for (int d = 0; d < b.spec_zone; ++d) {
    if (j == d || j == y_len - 1 - d) w = 1.0;
  }
  for (int d = b.spec_zone; d < b.relax_zone; ++d) {
    double linear = (b.relax_zone > 1) ? dmax(0.0, (double)(b.spec_zone + b.relax_zone - (d + 1)) / (double)(b.relax_zone - 1)) : 0.0;
    double weight = dmin(1.0, dmax(0.0, b.sub_ratio * 0.1 * linear));
    if (i >= d && i < x_len - d && (j == d || j == y_len - 1 - d)) w = weight;
  }
  return w;
}

// ---------------------------------------------------------------------------
// advance_uv, u faces (core/acoustic.py:626-735).
// ---------------------------------------------------------------------------
__global__ void k_advance_u(Grid g, Acoustic A, double dts, int top_lid, BdyArgs bdy) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny;
  if (i > nx || j >= ny) return;
  const int nxu = nx + 1;
  const size_t cu = ix3(k, j, i, ny, nxu);
  const size_t f2 = ix2(j, i, nxu);
  double u = A.u[cu] + dts * ld(A.u_tend, cu);
  const int l = (i == 0) ? 0 : i - 1;
  const int r = (i == nx) ? nx - 1 : i;
  auto P = [&](const double *a, int kk, int ic) { return ld(a, ix3(kk, j, ic, ny, nx)); };
  auto PH = [&](int kk, int ic) { return A.ph[ix3(kk, j, ic, ny, nx)]; };
  auto PP = [&](int kk, int ic) { return A.p[ix3(kk, j, ic, ny, nx)]; };
  auto AL = [&](int kk, int ic) { return A.al[ix3(kk, j, ic, ny, nx)]; };
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  const double ph_term = (PH(k + 1, r) - PH(k + 1, l)) + (PH(k, r) - PH(k, l));
  const double p_term = (P(A.alt, k, l) + P(A.alt, k, r)) * (PP(k, r) - PP(k, l));
  const double pb_term = (AL(k, l) + AL(k, r)) * (P(A.pb, k, r) - P(A.pb, k, l));
  const double mass_x = c1 * ld(A.muu, f2) + c2;
  const double msfr = ld(g.msfux, f2) / ld(g.msfuy, f2);
  double dpx = msfr * 0.5 * g.rdx * mass_x * (ph_term + p_term + pb_term);
  auto ps = [&](int m) { return PP(m, l) + PP(m, r); };
  const double mw_l = A.muts[ix2(j, l, nx)] - ld(A.mut, ix2(j, l, nx));
  const double mw_r = A.muts[ix2(j, r, nx)] - ld(A.mut, ix2(j, r, nx));
  const double bracket = ld(g.rdnw, k) * (dpn_acoustic(g, k + 1, top_lid, ps) - dpn_acoustic(g, k, top_lid, ps)) -
                         0.5 * (c1 * (mw_l + mw_r));
  dpx = dpx + msfr * g.rdx * (P(A.php, k, r) - P(A.php, k, l)) * bracket;
  u = u - dts * ld(A.cqu, cu) * dpx;
  const double md = -EMDIV * g.dx * (A.mudf[ix2(j, r, nx)] - A.mudf[ix2(j, l, nx)]) / ld(g.msfuy, f2);
  u = u + c1 * md;
  if (bdy.active) {
    const double w = relax_weight_u(j, i, ny, nxu, bdy);
    if (w != 0.0) u = u + w * (ld(bdy.u_target, cu) - u);
  }
  A.u[cu] = u;
}

// advance_uv, v faces (core/acoustic.py:737-750).
__global__ void k_advance_v(Grid g, Acoustic A, double dts, int top_lid, BdyArgs bdy) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny;
  if (i >= nx || j > ny) return;
  const int nyv = ny + 1;
  const size_t cv = ix3(k, j, i, nyv, nx);
  const size_t f2 = ix2(j, i, nx);
  double v = A.v[cv] + dts * ld(A.v_tend, cv);
  const int sj = (j == 0) ? 0 : j - 1;
  const int nj = (j == ny) ? ny - 1 : j;
  auto P = [&](const double *a, int kk, int jc) { return ld(a, ix3(kk, jc, i, ny, nx)); };
  auto PH = [&](int kk, int jc) { return A.ph[ix3(kk, jc, i, ny, nx)]; };
  auto PP = [&](int kk, int jc) { return A.p[ix3(kk, jc, i, ny, nx)]; };
  auto AL = [&](int kk, int jc) { return A.al[ix3(kk, jc, i, ny, nx)]; };
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  const double ph_term = (PH(k + 1, nj) - PH(k + 1, sj)) + (PH(k, nj) - PH(k, sj));
  const double p_term = (P(A.alt, k, sj) + P(A.alt, k, nj)) * (PP(k, nj) - PP(k, sj));
  const double pb_term = (AL(k, sj) + AL(k, nj)) * (P(A.pb, k, nj) - P(A.pb, k, sj));
  const double mass_y = c1 * ld(A.muv, f2) + c2;
  const double msfr = ld(g.msfvy, f2) / ld(g.msfvx, f2);
  double dpy = msfr * 0.5 * g.rdy * mass_y * (ph_term + p_term + pb_term);
  auto ps = [&](int m) { return PP(m, sj) + PP(m, nj); };
  const double mw_s = A.muts[ix2(sj, i, nx)] - ld(A.mut, ix2(sj, i, nx));
  const double mw_n = A.muts[ix2(nj, i, nx)] - ld(A.mut, ix2(nj, i, nx));
  const double bracket = ld(g.rdnw, k) * (dpn_acoustic(g, k + 1, top_lid, ps) - dpn_acoustic(g, k, top_lid, ps)) -
                         0.5 * (c1 * (mw_s + mw_n));
  dpy = dpy + msfr * g.rdy * (P(A.php, k, nj) - P(A.php, k, sj)) * bracket;
  v = v - dts * ld(A.cqv, cv) * dpy;
  const double md = -EMDIV * g.dy * (A.mudf[ix2(nj, i, nx)] - A.mudf[ix2(sj, i, nx)]) * (1.0 / ld(g.msfvx, f2));
  v = v + c1 * md;
  if (bdy.active) {
    const double w = relax_weight_v(j, i, nyv, nx, bdy);
    if (w != 0.0) v = v + w * (ld(bdy.v_target, cv) - v);
  }
  A.v[cv] = v;
}

// ---------------------------------------------------------------------------
// Column kernel: advance_mu_t + advance_w + calc_p_rho for one substep.
// ---------------------------------------------------------------------------
struct ColArgs {
  double dts, epssm;
  int specified, top_lid, w_damping, damp_opt;
  double dampcoef, zdamp;
};

__global__ void k_column(Grid g, Acoustic A, ColArgs c) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  const size_t c2d = ix2(j, i, nx);
  const double dts = c.dts;
  const double eps_p = 1.0 + c.epssm, eps_m = 1.0 - c.epssm;
  const double msftx = ld(g.msftx, c2d), msfty = ld(g.msfty, c2d);
  const double mut = ld(A.mut, c2d);
  auto M = [&](int k) { return ix3(k, j, i, ny, nx); };
  auto T1 = [&](int k, int jj, int ii2) { return ld(A.theta_s, ix3(k, jj, ii2, ny, nx)) - T0; };

  // ===================== advance_mu_t =====================
  const bool active = !c.specified || (j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2);
  if (active) {
    const int nxu = nx + 1, nyv = ny + 1;
    const double muv_n = ld(A.muv, ix2(j + 1, i, nx)), muv_s = ld(A.muv, ix2(j, i, nx));
    const double muu_e = ld(A.muu, ix2(j, i + 1, nxu)), muu_w = ld(A.muu, ix2(j, i, nxu));
    const double fvi_n = 1.0 / ld(g.msfvx, ix2(j + 1, i, nx)), fvi_s = 1.0 / ld(g.msfvx, ix2(j, i, nx));
    const double fuy_e = ld(g.msfuy, ix2(j, i + 1, nxu)), fuy_w = ld(g.msfuy, ix2(j, i, nxu));
    auto dvdxi_at = [&](int k) {
      const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
      const double vn = A.v[ix3(k, j + 1, i, nyv, nx)] + (c1 * muv_n + c2) * ld(A.v_1, ix3(k, j + 1, i, nyv, nx)) * fvi_n;
      const double vs = A.v[ix3(k, j, i, nyv, nx)] + (c1 * muv_s + c2) * ld(A.v_1, ix3(k, j, i, nyv, nx)) * fvi_s;
      const double ue = A.u[ix3(k, j, i + 1, ny, nxu)] + (c1 * muu_e + c2) * ld(A.u_1, ix3(k, j, i + 1, ny, nxu)) / fuy_e;
      const double uw = A.u[ix3(k, j, i, ny, nxu)] + (c1 * muu_w + c2) * ld(A.u_1, ix3(k, j, i, ny, nxu)) / fuy_w;
      return msftx * msfty * (g.rdy * (vn - vs) + g.rdx * (ue - uw));
    };
    double dmdt = 0.0;
    for (int k = 0; k < nz; ++k) {
      const double t = ld(g.dnw, k) * dvdxi_at(k);
      dmdt = (k == 0) ? t : dmdt + t;
    }
    const double mu_work_old = A.muts[c2d] - mut;
    const double mu_save = A.mu[c2d] - mu_work_old;
    double mu_tend = (A.mu_tend != nullptr) ? ld(A.mu_tend, c2d) : 0.0;
    double mu_tendency = dmdt + mu_tend;
    double scale = 1.0;
    if (c.specified) {
      const double floor_ = dmax(MIN_MUTS_PA, MIN_MUTS_FRACTION * mut);
      const double muts_old = mut + mu_work_old;
      const double raw = dts * mu_tendency;
      const double allowed = dmax(muts_old - floor_, 0.0);
      const double loss = -raw;
      const bool finite = isfinite(raw) && isfinite(muts_old);
      scale = (finite && (loss > allowed)) ? allowed / dmax(loss, 1.0) : (finite ? 1.0 : 0.0);
      scale = dmin(dmax(scale, 0.0), 1.0);
      mu_tendency = mu_tendency * scale;
      dmdt = dmdt * scale;
      mu_tend = mu_tend * scale;
    }
    const double mu_work_new = mu_work_old + dts * mu_tendency;
    A.mu[c2d] = mu_save + mu_work_new;
    A.mudf[c2d] = mu_tendency;
    A.muts[c2d] = mut + mu_work_new;
    A.muave[c2d] = 0.5 * ((1.0 + c.epssm) * mu_work_new + (1.0 - c.epssm) * mu_work_old);
    // ww recurrence (face 0 keeps ww(0) - ww_1(0); face nz keeps ww(nz)).
    double prev = A.ww[M(0)];
    A.ww[M(0)] = prev - ld(A.ww_1, M(0));
    for (int kk = 1; kk < nz; ++kk) {
      const int k = kk - 1;
      double dv = dvdxi_at(k);
      if (c.specified) dv = dv * scale;
      const double inc = ld(g.dnw, k) * (ld(g.c1h, k) * dmdt + dv + ld(g.c1h, k) * mu_tend) / msfty;
      const double cur = prev - inc;
      A.ww[M(kk)] = cur - ld(A.ww_1, M(kk));
      prev = cur;
    }
    // theta work update with wdtn
    int ie, iw, jn, js;
    if (c.specified) {
      ie = i + 1; iw = i - 1; jn = j + 1; js = j - 1;
    } else {
      ie = wrp(i + 1, nx); iw = wrp(i - 1, nx); jn = wrp(j + 1, ny); js = wrp(j - 1, ny);
    }
    double wdtn_lo = 0.0;
    for (int k = 0; k < nz; ++k) {
      double wdtn_hi = 0.0;
      if (k + 1 <= nz - 1) {
        wdtn_hi = A.ww[M(k + 1)] * (ld(g.fnm, k + 1) * T1(k + 1, j, i) + ld(g.fnp, k + 1) * T1(k, j, i));
      }
      const double th = T1(k, j, i);
      const double v_flux = A.v[ix3(k, j + 1, i, nyv, nx)] * (T1(k, jn, i) + th) - A.v[ix3(k, j, i, nyv, nx)] * (th + T1(k, js, i));
      const double u_flux = A.u[ix3(k, j, i + 1, ny, nxu)] * (T1(k, j, ie) + th) - A.u[ix3(k, j, i, ny, nxu)] * (th + T1(k, j, iw));
      const double tend = msftx * (0.5 * g.rdy * v_flux + 0.5 * g.rdx * u_flux) + ld(g.rdnw, k) * (wdtn_hi - wdtn_lo);
      const double theta_i = A.theta_w[M(k)] + msfty * dts * ld(A.t_tend, M(k));
      A.theta_w[M(k)] = theta_i - dts * msfty * tend;
      wdtn_lo = wdtn_hi;
    }
  }

  // ===================== advance_w =====================
  const double muts = A.muts[c2d];
  const double muave = A.muave[c2d];
  const double minv = 1.0 / msfty;
  auto mass_h_muts = [&](int k) { return ld(g.c1h, k) * muts + ld(g.c2h, k); };
  auto mass_f_mut = [&](int k) { return ld(g.c1f, k) * mut + ld(g.c2f, k); };
  auto mass_f_muts = [&](int k) { return ld(g.c1f, k) * muts + ld(g.c2f, k); };
  auto coef = [&](int k) { return ld(A.c2a, M(k)) * ld(g.rdnw, k) / safe12(ld(g.c1h, k) * mut + ld(g.c2h, k)); };
  auto t2a_at = [&](int k) {
    const double half = 0.5 * (eps_p * A.theta_w[M(k)] + eps_m * A.t2ave[M(k)]);
    return (half + (ld(g.c1h, k) * muave) * T0) / (mass_h_muts(k) * (T0 + T1(k, j, i)));
  };
  auto wd = [&](int m) {  // phi advection wdwn on mass level m
    const double wwm = 0.5 * (A.ww[M(m + 1)] + A.ww[M(m)]);
    return wwm * ld(g.rdnw, m) * (ld(A.pt1, M(m + 1)) - ld(A.pt1, M(m)));
  };
  const double c05gem = 0.5 * G * eps_m;
  auto rhs_at = [&](int f, double wd_f, double wd_fm1) {  // f in 1..nz
    double r = dts * (ld(A.ph_tend, M(f)) + c05gem * A.w[M(f)]);
    if (f < nz) r = r + (-(dts * (ld(g.fnm, f) * wd_f + ld(g.fnp, f) * wd_fm1)));
    r = A.ph[M(f)] + msfty * r / mass_f_mut(f);
    if (f == nz && c.top_lid) r = 0.0;
    return r;
  };
  // terrain surface w (u_1, v_1 decoupled stage winds; ht edge-padded)
  double w_surface;
  {
    auto HT = [&](int jj, int ii2) {
      jj = jj < 0 ? 0 : (jj > ny - 1 ? ny - 1 : jj);
      ii2 = ii2 < 0 ? 0 : (ii2 > nx - 1 ? nx - 1 : ii2);
      return ld(A.phb0, ix2(jj, ii2, nx)) / G;
    };
    const double htc = HT(j, i);
    const double dy_n = HT(j + 1, i) - htc, dy_s = htc - HT(j - 1, i);
    const double dx_e = HT(j, i + 1) - htc, dx_w = htc - HT(j, i - 1);
    auto vcf = [&](int jv) {
      return g.cf1 * ld(A.v_1, ix3(0, jv, i, ny + 1, nx)) + g.cf2 * ld(A.v_1, ix3(1, jv, i, ny + 1, nx)) +
             g.cf3 * ld(A.v_1, ix3(2, jv, i, ny + 1, nx));
    };
    auto ucf = [&](int iu) {
      return g.cf1 * ld(A.u_1, ix3(0, j, iu, ny, nx + 1)) + g.cf2 * ld(A.u_1, ix3(1, j, iu, ny, nx + 1)) +
             g.cf3 * ld(A.u_1, ix3(2, j, iu, ny, nx + 1));
    };
    w_surface = msfty * 0.5 * g.rdy * (dy_n * vcf(j + 1) + dy_s * vcf(j)) +
                msftx * 0.5 * g.rdx * (dx_e * ucf(i + 1) + dx_w * ucf(i));
  }
  // Upward sweep: explicit w update and Thomas forward elimination.  The
  // forward-swept w is stored in A.w and the phi predictor rhs in A.ph (the
  // old values are consumed in this sweep before being overwritten).
  const double c05dg = 0.5 * dts * G;
  const double dtsg = dts * G;
  double wf_prev = w_surface;
  A.w[M(0)] = w_surface;
  // rolling window
  double rhs_m1 = 0.0;                      // rhs(f-1), rhs(0) = 0
  double wd_0 = wd(0);
  double wd_1 = (nz >= 2) ? wd(1) : 0.0;
  double rhs_0 = rhs_at(1, wd_1, wd_0);     // rhs(1)
  double ph_m1 = A.ph[M(0)], ph_0 = A.ph[M(1)];
  double t2a_m1 = t2a_at(0);
  double buoy_m1 = ld(A.c2a, M(0)) * ld(A.alt, M(0)) * t2a_m1;
  double coef_m1 = coef(0);
  A.t2ave[M(0)] = t2a_m1;
  double wd_prev = wd_1;  // wd(f)
  for (int f = 1; f <= nz; ++f) {
    double w_next;
    const double w_old = A.w[M(f)];
    if (f < nz) {
      const double wd_next = (f + 1 <= nz - 1) ? wd(f + 1) : 0.0;
      const double rhs_p1 = rhs_at(f + 1, wd_next, wd_prev);
      const double ph_p1 = A.ph[M(f + 1)];
      const double t2a_f = t2a_at(f);
      A.t2ave[M(f)] = t2a_f;
      const double buoy_f = ld(A.c2a, M(f)) * ld(A.alt, M(f)) * t2a_f;
      const double coef_f = coef(f);
      double rw = ld(A.rw_tend, M(f));
      if (c.w_damping == 1) {
        const double mf = ld(g.c1f, f) * mut + ld(g.c2f, f);
        const double vert_cfl = fabs(A.ww[M(f)] / safe12(mf) * ld(g.rdnw, f) * dts);
        double damp = -sgn(w_old) * W_ALPHA * (vert_cfl - W_BETA) * mf;
        damp = (vert_cfl > W_BETA) ? damp : 0.0;
        rw = rw + damp;
      }
      w_next = w_old + dts * rw;
      const double tA_u = coef_f * (eps_p * (rhs_p1 - rhs_0) + eps_m * (ph_p1 - ph_0));
      const double tA_l = coef_m1 * (eps_p * (rhs_0 - rhs_m1) + eps_m * (ph_0 - ph_m1));
      const double tA = minv * ld(A.cqw, M(f)) * (c05dg * ld(g.rdn, f)) * (tA_u - tA_l);
      const double tB = dtsg * minv * (ld(g.rdn, f) * (buoy_f - buoy_m1) - (ld(g.c1f, f) * muave));
      w_next = w_next + (tA + tB);
      // shift the window
      A.ph[M(f - 1)] = (f - 1 == 0) ? ph_m1 : rhs_m1;  // store rhs(f-1) for the back sweep
      rhs_m1 = rhs_0;
      rhs_0 = rhs_p1;
      ph_m1 = ph_0;
      ph_0 = ph_p1;
      buoy_m1 = buoy_f;
      coef_m1 = coef_f;
      wd_prev = wd_next;
    } else {
      // top face (rhs_0 = rhs(nz), rhs_m1 = rhs(nz-1), ph_0 = ph(nz), ph_m1 = ph(nz-1))
      const int km1 = nz - 1;
      const double mhm = safe12(ld(g.c1h, km1) * mut + ld(g.c2h, km1));
      const double rdnw_t = ld(g.rdnw, km1);
      const double t2a_t = A.t2ave[M(km1)];
      const double tA_top = -0.5 * dts * G / mhm * (rdnw_t * rdnw_t) * 2.0 * ld(A.c2a, M(km1)) *
                            (eps_p * (rhs_0 - rhs_m1) + eps_m * (ph_0 - ph_m1));
      const double tB_top = -dts * G * (2.0 * rdnw_t * ld(A.c2a, M(km1)) * ld(A.alt, M(km1)) * t2a_t + (ld(g.c1f, nz) * muave));
      const double w_top = w_old + dts * ld(A.rw_tend, M(nz)) + minv * (tA_top + tB_top);
      w_next = c.top_lid ? 0.0 : w_top;
      A.ph[M(nz - 1)] = rhs_m1;  // rhs(nz-1)
      A.ph[M(nz)] = rhs_0;       // rhs(nz)
    }
    const double wf = (w_next - ld(A.a, M(f)) * wf_prev) * ld(A.alpha, M(f));
    A.w[M(f)] = wf;
    wf_prev = wf;
  }
  // A.ph now holds: ph(0) at face 0 (unchanged), rhs(f) at faces 1..nz.
  // Downward sweep: back substitution, Rayleigh damping, phi finish and
  // calc_p_rho on the mass level below each face.
  double dampmag = 0.0, htop = 0.0, hbot = 0.0;
  const bool do_damp = (c.damp_opt == 3 && c.dampcoef > 0.0);
  if (do_damp) {
    dampmag = dts * c.dampcoef;
    htop = ld(A.pt1, M(nz)) / G;
    hbot = htop - c.zdamp;
  }
  auto damp_face = [&](int f, double ws) {
    if (!do_damp) return ws;
    const double hk = ld(A.pt1, M(f)) / G;
    const double sv = sin(0.5 * 3.141592653589793 * (hk - hbot) / c.zdamp);
    const double ramp = sv * sv;
    const double dampwt = (hk >= hbot) ? dampmag * ramp : 0.0;
    return (ws - dampwt * mass_f_mut(f) * ld(A.w_save, M(f))) / (1.0 + dampwt);
  };
  const double mu_work = muts - mut;
  double ws_next = A.w[M(nz)];  // wf(nz)
  double ph_up;                 // ph_next(f+1)
  {
    const double ws_top = damp_face(nz, ws_next);
    A.w[M(nz)] = ws_top;
    const double rhs_t = A.ph[M(nz)];
    ph_up = rhs_t + msfty * 0.5 * dts * G * eps_p * ws_top / mass_f_muts(nz);
    A.ph[M(nz)] = ph_up;
  }
  for (int f = nz - 1; f >= 0; --f) {
    double ph_f;
    if (f >= 1) {
      const double wsf = A.w[M(f)] - ld(A.gamma, M(f)) * ws_next;
      ws_next = wsf;  // undamped value feeds the next back-substitution step
      const double wsd = damp_face(f, wsf);
      A.w[M(f)] = wsd;
      ph_f = A.ph[M(f)] + msfty * 0.5 * dts * G * eps_p * wsd / mass_f_muts(f);
      A.ph[M(f)] = ph_f;
    } else {
      ph_f = A.ph[M(0)];
    }
    // calc_p_rho on mass level f (needs ph_next(f), ph_next(f+1))
    const int k = f;
    const double mass = ld(g.c1h, k) * muts + ld(g.c2h, k);
    const double safe = safe12(mass);
    const double mu_term = ld(g.c1h, k) * mu_work;
    const double altc = ld(A.alt, M(k));
    const double al = -(altc * mu_term + ld(g.rdnw, k) * (ph_up - ph_f)) / safe;
    const double t1 = T1(k, j, i);
    const double ttr = T0 + t1;
    const double sttr = fabs(ttr) > 1.0e-6 ? ttr : 1.0e-6;
    const double pp = ld(A.c2a, M(k)) * (altc * (A.theta_w[M(k)] - mu_term * t1) / (safe * sttr) - al);
    const double pm1 = A.pm1[M(k)];
    A.p[M(k)] = pp + SMDIV * (pp - pm1);
    A.pm1[M(k)] = pp;
    A.al[M(k)] = al;
    ph_up = ph_f;
  }
}

}  // namespace wg
