// Column kernel of one acoustic substep, one thread per column.
//
// advance_mu_t (dynamics/mu_t_advance.py:131-451), advance_w with its Thomas
// solve (core/advance_w.py:293-627) and calc_p_rho with smdiv memory
// (core/calc_p_rho.py:137-183) for one column (i, j), in three sweeps over
// the levels that carry every recurrence in registers:
//   sweep 1 (up)   dmdt = sum_k dnw*dvdxi and the 2-D mass update;
//   sweep 2 (up)   the ww prefix, the theta update and t_2ave, the phi
//                  predictor rhs, the explicit w and the Thomas forward
//                  elimination, each one or two levels behind the level
//                  whose loads are in flight;
//   sweep 3 (down) Thomas back substitution, Rayleigh damping, w and phi
//                  out, and calc_p_rho one level behind.
// The inputs of each iteration are loaded several iterations ahead into a
// ring of register buffers (3 levels up, 4 faces down, the column sum 8-16
// levels), so every thread keeps dozens of loads in flight with no block
// barrier anywhere;
// the forward-elimination result and the phi predictor of each face are
// parked in warp-private shared memory for sweep 3 (2 (nz+1) doubles per
// column).  A warp owns 32 adjacent columns of one row, so every load and
// store of a level is one coalesced 256-byte row segment.
//
// Every expression, and the order of every sum and recurrence, is the
// level-parallel kernel's (column_tiled.cuh) and the reference's, so the
// results are identical bit for bit.
#pragma once
#include "dycore_common.cuh"
#include "acoustic_kernels.cuh"

namespace wg {

// Warps per block (each one row segment of 32 columns); two blocks per SM.
#ifndef WG_CS_WARPS
#define WG_CS_WARPS 4
#endif
constexpr int CS_WARPS = WG_CS_WARPS;

inline size_t column_stream_smem_bytes(int nz) { return (size_t)2 * (nz + 1) * 32 * CS_WARPS * sizeof(double); }

// Coherent load of an array this kernel also writes.
__device__ __forceinline__ double ldw(const double *p, size_t i) { return p[i]; }

template <bool PIN = false>
__global__ void __launch_bounds__(32 * CS_WARPS, 2) k_column_stream(Grid g, Acoustic A, ColArgs c,
                                                                      const double *dvdxi, const double *hdiv) {
  extern __shared__ double sm[];
  const int lane = threadIdx.x, wid = threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz, L = nz + 1;
  const int i = blockIdx.x * 32 + lane;
  const int j = blockIdx.y * CS_WARPS + wid;
  if (i >= nx || j >= ny) return;
  // warp-private scratch: forward-eliminated w and the phi predictor per face
  double *s_wf = sm + (size_t)wid * 2 * L * 32 + lane;
  double *s_rhs = s_wf + (size_t)L * 32;
  auto WF = [&](int f) -> double & { return s_wf[(size_t)f * 32]; };
  auto RHS = [&](int f) -> double & { return s_rhs[(size_t)f * 32]; };

  const int plane = ny * nx;
  const size_t c2d = ix2(j, i, nx);
  const size_t m0 = c2d;  // offset of level 0; level k adds k * plane
  auto M = [&](int k) { return m0 + (size_t)(unsigned)(k * plane); };
  const double dts = c.dts;
  const double eps_p = 1.0 + c.epssm, eps_m = 1.0 - c.epssm;
  const double msftx = ld(g.msftx, c2d);
  const double msfty = ld(g.msfty, c2d);
  const double mut = ld(A.mut, c2d);
  const double minv = ld(g.rmsfty, c2d);  // == 1.0 / msfty
  const bool active = !c.specified || (j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2);
  const int nxu = nx + 1, nyv = ny + 1;

  // ------------------------------------------------------------------
  // sweep 1: dmdt and the 2-D mass update (advance_mu_t)
  // ------------------------------------------------------------------
  double dmdt = 0.0, mu_tend = 0.0, scale = 1.0, muts, muave;
  const double ww_bot = ldw(A.ww, M(0)), ww_top = ldw(A.ww, M(nz));
  if (active) {
    const double muts_in = ldw(A.muts, c2d);
    const double mu_in = ldw(A.mu, c2d);
    mu_tend = (A.mu_tend != nullptr) ? ld(A.mu_tend, c2d) : 0.0;
    // the column sum in level order, its loads batched SB levels ahead
    constexpr int SB = 8;
    double ba[SB], bb[SB];
    auto ldb = [&](int k0, double *b) {
#pragma unroll
      for (int u = 0; u < SB; ++u) b[u] = (k0 + u < nz) ? ld(dvdxi, M(k0 + u)) : 0.0;
    };
    auto acc = [&](int k0, const double *b) {
#pragma unroll
      for (int u = 0; u < SB; ++u) {
        if (k0 + u < nz) {
          const double t = ld(g.dnw, k0 + u) * b[u];
          dmdt = (k0 + u == 0) ? t : dmdt + t;
        }
      }
    };
    ldb(0, ba);
    for (int k0 = 0; k0 < nz; k0 += 2 * SB) {
      ldb(k0 + SB, bb);
      acc(k0, ba);
      ldb(k0 + 2 * SB, ba);
      acc(k0 + SB, bb);
    }
    const double mu_work_old = muts_in - mut;
    const double mu_save = mu_in - mu_work_old;
    double mu_tendency = dmdt + mu_tend;
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
    muts = mut + mu_work_new;
    muave = 0.5 * ((1.0 + c.epssm) * mu_work_new + (1.0 - c.epssm) * mu_work_old);
    A.mu[c2d] = mu_save + mu_work_new;
    A.mudf[c2d] = mu_tendency;
    A.muts[c2d] = muts;
    A.muave[c2d] = muave;
  } else if (PIN && c.cad) {
    // specified cadence: ring-0 mu', muts and muave pinned to the mu' leaf
    const double mu_pin = ring_target(c.cad_mu, 1, ny, nx, 0, j, i);
    const double muts_pin = ld(c.mub, c2d) + mu_pin;
    muts = muts_pin;
    muave = muts_pin - mut;
    A.mu[c2d] = mu_pin;
    A.muts[c2d] = muts;
    A.muave[c2d] = muave;
  } else {
    muts = ldw(A.muts, c2d);
    muave = ldw(A.muave, c2d);
  }

  // ------------------------------------------------------------------
  // explicit w at the surface (face 0): terrain slope times the
  // extrapolated decoupled u_1 / v_1 (core/advance_w.py via acoustic.py:976-1002)
  // ------------------------------------------------------------------
  double wn0;
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
      return g.cf1 * ld(A.v_1, ix3(0, jv, i, nyv, nx)) + g.cf2 * ld(A.v_1, ix3(1, jv, i, nyv, nx)) +
             g.cf3 * ld(A.v_1, ix3(2, jv, i, nyv, nx));
    };
    auto ucf = [&](int iu) {
      return g.cf1 * ld(A.u_1, ix3(0, j, iu, ny, nxu)) + g.cf2 * ld(A.u_1, ix3(1, j, iu, ny, nxu)) +
             g.cf3 * ld(A.u_1, ix3(2, j, iu, ny, nxu));
    };
    wn0 = msfty * 0.5 * g.rdy * (dy_n * vcf(j + 1) + dy_s * vcf(j)) +
          msftx * 0.5 * g.rdx * (dx_e * ucf(i + 1) + dx_w * ucf(i));
  }

  // ------------------------------------------------------------------
  // sweep 2 (up).  Iteration k: ww at face k+1 (prefix), the theta /
  // t_2ave / buoyancy / coef / wd of level k, the phi predictor of face k,
  // then the explicit w and the forward elimination of face k-1.
  // ------------------------------------------------------------------
  // per-iteration inputs: iteration k reads face k, level k and the three
  // values of k+1 its stencils reach (ww_1, theta, pt1), loaded LA2 = 3
  // iterations ahead into a ring of four buffers
  struct In {
    double dv, hd, thw, ttend, t2o, c2a, alt, ph, pht, w, rwt, cqw, a, alpha, ww1n, thn, pt1n;
  };
  auto load = [&](int k, In &v) {
    const size_t o = M(k);
    v.ph = ldw(A.ph, o);
    v.pht = ld(A.ph_tend, o);
    v.w = ldw(A.w, o);
    v.rwt = ld(A.rw_tend, o);
    v.cqw = ld(A.cqw, o);
    v.a = ld(A.a, o);
    v.alpha = ld(A.alpha, o);
    if (k < nz) {
      const size_t o1 = M(k + 1);
      v.dv = active ? ld(dvdxi, o) : 0.0;
      v.hd = active ? ld(hdiv, o) : 0.0;
      v.thw = ldw(A.theta_w, o);
      v.ttend = ld(A.t_tend, o);
      v.t2o = ldw(A.t2ave, o);
      v.c2a = ld(A.c2a, o);
      v.alt = ld(A.alt, o);
      v.ww1n = ld(A.ww_1, o1);
      v.pt1n = ld(A.pt1, o1);
      v.thn = (k + 1 < nz) ? ld(A.theta_s, o1) - T0 : 0.0;
    }
  };
  In b0, b1, b2, b3;
  load(0, b0);
  load(1, b1);
  load(2, b2);
  const double ww1_0 = ld(A.ww_1, M(0));
  double th_k = ld(A.theta_s, M(0)) - T0;  // theta' at level k (the window)
  double pt1_k = ld(A.pt1, M(0));          // pt1 at face k

  const double c05gem = 0.5 * G * eps_m;
  const double c05dg = 0.5 * dts * G;
  const double dtsg = dts * G;
  // ww prefix state: ww at faces k and k+1, the running sum `prev`
  double prev = ww_bot;
  double ww_k = active ? (ww_bot - ww1_0) : ww_bot;  // face 0 (inactive: old ww)
  // windows of the level / face quantities the later stencils read
  double thm1 = 0.0;                    // T1 at level k-1
  double wd_m1 = 0.0;                   // wd at level k-1
  double coef_m1 = 0.0, coef_m2 = 0.0;  // coef at levels k-1, k-2
  double buoy_m1 = 0.0, buoy_m2 = 0.0;  // buoyancy at levels k-1, k-2
  double rhs_m1 = 0.0, rhs_m2 = 0.0;    // phi predictor at faces k-1, k-2
  double ph_m1 = 0.0, ph_m2 = 0.0;      // old phi at faces k-1, k-2
  double ww_m1 = 0.0;                   // ww at face k-1
  double w_m1 = 0.0, rwt_m1 = 0.0, cqw_m1 = 0.0, a_m1 = 0.0, alpha_m1 = 0.0;  // face k-1 inputs
  double t2a_m1 = 0.0, c2a_m1 = 0.0, alt_m1 = 0.0;                            // level k-1 (top face)
  double wf_prev = 0.0;                 // forward-eliminated w at face k-2

  // one iteration; the four input buffers rotate by unrolling the loop four
  // ways (a register copy of a buffer would wait for its loads)
  auto step2 = [&](int k, const In &cur, In &nx3) {
    if (k + 3 <= nz) load(k + 3, nx3);
    // --- ww at face k+1 (advance_mu_t's ww prefix, mu_t_advance.py:229-237) ---
    double ww_k1 = 0.0;
    if (k + 1 <= nz) {
      if (!active) {
        ww_k1 = ldw(A.ww, M(k + 1));
      } else if (k + 1 == nz) {
        ww_k1 = ww_top;
      } else {
        const int kl = k;  // increment of face k+1 uses level k
        double dv = cur.dv;
        if (c.specified) dv = dv * scale;
        const double inc =
            div_rcp(ld(g.dnw, kl) * (ld(g.c1h, kl) * dmdt + dv + ld(g.c1h, kl) * mu_tend), msfty, minv);
        const double cc = prev - inc;
        ww_k1 = cc - cur.ww1n;
        prev = cc;
      }
    }
    if (active) A.ww[M(k)] = ww_k;

    // --- level k: theta update, t_2ave, buoyancy, coef, wd (P5) ---
    double wd_k = 0.0, coef_k = 0.0, buoy_k = 0.0, t2a_k = 0.0;
    if (k < nz) {
      const double th_p1 = (k + 1 < nz) ? cur.thn : 0.0;
      double thw = cur.thw;
      if (active) {
        const double wdtn_hi = (k + 1 <= nz - 1) ? ww_k1 * (ld(g.fnm, k + 1) * th_p1 + ld(g.fnp, k + 1) * th_k) : 0.0;
        const double wdtn_lo = (k >= 1) ? ww_k * (ld(g.fnm, k) * th_k + ld(g.fnp, k) * thm1) : 0.0;
        const double tend = cur.hd + ld(g.rdnw, k) * (wdtn_hi - wdtn_lo);
        const double theta_i = thw + msfty * dts * cur.ttend;
        thw = theta_i - dts * msfty * tend;
        A.theta_w[M(k)] = thw;
      } else if (PIN && c.cad) {
        // specified cadence: the ring-0 work theta whose finished theta is the leaf's
        const double mass_pin = ld(g.c1h, k) * muts + ld(g.c2h, k);
        const double mass_cur = ld(g.c1h, k) * mut + ld(g.c2h, k);
        thw = mass_pin * (ring_target(c.cad_th, nz, ny, nx, k, j, i) - T0) - mass_cur * th_k;
        A.theta_w[M(k)] = thw;
      }
      const double mass_h = ld(g.c1h, k) * muts + ld(g.c2h, k);
      const double half = 0.5 * (eps_p * thw + eps_m * cur.t2o);
      t2a_k = (half + (ld(g.c1h, k) * muave) * T0) / (mass_h * (T0 + th_k));
      A.t2ave[M(k)] = t2a_k;
      buoy_k = cur.c2a * cur.alt * t2a_k;
      coef_k = cur.c2a * ld(g.rdnw, k) / safe12(ld(g.c1h, k) * mut + ld(g.c2h, k));
      const double wwm = 0.5 * (ww_k1 + ww_k);
      wd_k = wwm * ld(g.rdnw, k) * (cur.pt1n - pt1_k);
    }

    // --- face k: the phi predictor (P6) ---
    double rhs_k;
    if (k == 0) {
      rhs_k = 0.0;
    } else {
      double r = dts * (cur.pht + c05gem * cur.w);
      if (k < nz) r = r + (-(dts * (ld(g.fnm, k) * wd_k + ld(g.fnp, k) * wd_m1)));
      const double mf = ld(g.c1f, k) * mut + ld(g.c2f, k);
      r = cur.ph + msfty * r / mf;
      if (k == nz && c.top_lid) r = 0.0;
      rhs_k = r;
    }
    RHS(k) = rhs_k;

    // --- face f = k-1: explicit w (P7) and forward elimination (P8) ---
    if (k >= 1) {
      const int f = k - 1;
      double wn;
      if (f == 0) {
        wn = wn0;
      } else {
        const double w_old = w_m1;
        double rw = rwt_m1;
        if (c.w_damping == 1) {
          const double mf = ld(g.c1f, f) * mut + ld(g.c2f, f);
          const double vert_cfl = fabs(ww_m1 / safe12(mf) * ld(g.rdnw, f) * dts);
          double damp = -sgn(w_old) * W_ALPHA * (vert_cfl - W_BETA) * mf;
          damp = (vert_cfl > W_BETA) ? damp : 0.0;
          rw = rw + damp;
        }
        wn = w_old + dts * rw;
        const double tA_u = coef_m1 * (eps_p * (rhs_k - rhs_m1) + eps_m * (cur.ph - ph_m1));
        const double tA_l = coef_m2 * (eps_p * (rhs_m1 - rhs_m2) + eps_m * (ph_m1 - ph_m2));
        const double tA = minv * cqw_m1 * (c05dg * ld(g.rdn, f)) * (tA_u - tA_l);
        const double tB = dtsg * minv * (ld(g.rdn, f) * (buoy_m1 - buoy_m2) - (ld(g.c1f, f) * muave));
        wn = wn + (tA + tB);
      }
      const double wf = (f == 0) ? wn : (wn - a_m1 * wf_prev) * alpha_m1;
      WF(f) = wf;
      wf_prev = wf;
    }

    // --- slide the windows ---
    if (k < nz) {
      thm1 = th_k;
      th_k = cur.thn;
      pt1_k = cur.pt1n;
    }
    wd_m1 = wd_k;
    coef_m2 = coef_m1; coef_m1 = coef_k;
    buoy_m2 = buoy_m1; buoy_m1 = buoy_k;
    rhs_m2 = rhs_m1; rhs_m1 = rhs_k;
    ph_m2 = ph_m1; ph_m1 = cur.ph;
    ww_m1 = ww_k;
    w_m1 = cur.w; rwt_m1 = cur.rwt; cqw_m1 = cur.cqw; a_m1 = cur.a; alpha_m1 = cur.alpha;
    if (k < nz) {
      t2a_m1 = t2a_k; c2a_m1 = cur.c2a; alt_m1 = cur.alt;
    }
    ww_k = ww_k1;
  };
  for (int k = 0; k <= nz; k += 4) {
    step2(k, b0, b3);
    if (k + 1 <= nz) step2(k + 1, b1, b0);
    if (k + 2 <= nz) step2(k + 2, b2, b1);
    if (k + 3 <= nz) step2(k + 3, b3, b2);
  }
  // --- face nz: the top explicit w and its forward elimination ---
  {
    const int km1 = nz - 1;
    const double mhm = safe12(ld(g.c1h, km1) * mut + ld(g.c2h, km1));
    const double rdnw_t = ld(g.rdnw, km1);
    // after the loop: rhs_m1 = rhs(nz), rhs_m2 = rhs(nz-1); ph_m1 = ph(nz), ph_m2 = ph(nz-1);
    // w_m1 / rwt_m1 / a_m1 / alpha_m1 are face nz's inputs; t2a_m1 / c2a_m1 / alt_m1 level nz-1's
    const double tA_top = -0.5 * dts * G / mhm * (rdnw_t * rdnw_t) * 2.0 * c2a_m1 *
                          (eps_p * (rhs_m1 - rhs_m2) + eps_m * (ph_m1 - ph_m2));
    const double tB_top = -dts * G * (2.0 * rdnw_t * c2a_m1 * alt_m1 * t2a_m1 + (ld(g.c1f, nz) * muave));
    const double w_top = w_m1 + dts * rwt_m1 + minv * (tA_top + tB_top);
    const double wn = c.top_lid ? 0.0 : w_top;
    const double wf = (wn - a_m1 * wf_prev) * alpha_m1;
    WF(nz) = wf;
  }

  // ------------------------------------------------------------------
  // sweep 3 (down): back substitution, damping, w and phi out (P8b, P9),
  // calc_p_rho at level f once phi of faces f and f+1 are final (P10)
  // ------------------------------------------------------------------
  const bool do_damp = (c.damp_opt == 3 && c.dampcoef > 0.0);
  double dampmag = 0.0, hbot = 0.0;
  if (do_damp) {
    dampmag = dts * c.dampcoef;
    hbot = div_rcp(ld(A.pt1, M(nz)), G, RG) - c.zdamp;
  }
  const double mu_work = muts - mut;
  double ws_next = 0.0;    // undamped back-substituted w at face f+1
  double phn_up = 0.0;     // final phi at face f+1
  // face-f inputs of the back substitution and damping, and level-f inputs
  // of calc_p_rho, loaded four faces ahead (downward) into a ring of five
  struct In3 {
    double gm, pt, wsv, thw, alt, c2a, th, pm1;
  };
  auto load3 = [&](int f, In3 &v) {
    const size_t o = M(f);
    v.gm = (f >= 1 && f <= nz - 1) ? ld(A.gamma, o) : 0.0;
    v.pt = (do_damp && f >= 1) ? ld(A.pt1, o) : 0.0;
    v.wsv = (do_damp && f >= 1) ? ld(A.w_save, o) : 0.0;
    if (f < nz) {
      v.thw = ldw(A.theta_w, o);
      v.alt = ld(A.alt, o);
      v.c2a = ld(A.c2a, o);
      v.th = ld(A.theta_s, o) - T0;
      v.pm1 = ldw(A.pm1, o);
    }
  };
  auto step3 = [&](int f, const In3 &cur, In3 &nx4) {
    if (f - 4 >= 0) load3(f - 4, nx4);
    // back substitution (undamped), core/advance_w.py:583-592
    double ws;
    if (f == nz || f == 0) {
      ws = WF(f);
    } else {
      ws = WF(f) - cur.gm * ws_next;
    }
    ws_next = ws;
    // P9: damping, w and phi out
    double phn;
    if (f >= 1) {
      if (do_damp) {
        const double hk = div_rcp(cur.pt, G, RG);
        const double sv = sin(over_zdamp(0.5 * 3.141592653589793 * (hk - hbot), c));
        const double ramp = sv * sv;
        const double dampwt = (hk >= hbot) ? dampmag * ramp : 0.0;
        const double mf = ld(g.c1f, f) * mut + ld(g.c2f, f);
        ws = (ws - dampwt * mf * cur.wsv) / (1.0 + dampwt);
      }
      const double mfs = ld(g.c1f, f) * muts + ld(g.c2f, f);
      phn = RHS(f) + msfty * 0.5 * dts * G * eps_p * ws / mfs;
    } else {
      phn = ldw(A.ph, M(0));  // face 0 keeps the old phi
    }
    if (PIN && !active && c.ph_pin) {
      // ring-0 work ph whose finished ph' is the leaf's (spec_bdyupdate_ph)
      phn = ring_target(c.cad_ph, nz + 1, ny, nx, f, j, i) - ld(c.ph_save, M(f));
    }
    if (f >= 1 || (PIN && !active && c.ph_pin)) A.ph[M(f)] = phn;
    A.w[M(f)] = ws;
    // P10: calc_p_rho with smdiv memory at level f (faces f and f+1 final)
    if (f <= nz - 1) {
      const int k = f;
      const double mass = ld(g.c1h, k) * muts + ld(g.c2h, k);
      const double safe = safe12(mass);
      const double mu_term = ld(g.c1h, k) * mu_work;
      const double altc = cur.alt;
      const double al = -(altc * mu_term + ld(g.rdnw, k) * (phn_up - phn)) / safe;
      const double t1 = cur.th;
      const double ttr = T0 + t1;
      const double sttr = fabs(ttr) > 1.0e-6 ? ttr : 1.0e-6;
      const double pp = cur.c2a * (altc * (cur.thw - mu_term * t1) / (safe * sttr) - al);
      A.p[M(k)] = pp + SMDIV * (pp - cur.pm1);
      A.pm1[M(k)] = pp;
      A.al[M(k)] = al;
    }
    phn_up = phn;
  };
  In3 x0, x1, x2, x3, x4;
  load3(nz, x0);
  load3(nz - 1, x1);
  load3(nz - 2, x2);
  load3(nz - 3, x3);
  for (int f = nz; f >= 0; f -= 5) {
    step3(f, x0, x4);
    if (f - 1 >= 0) step3(f - 1, x1, x0);
    if (f - 2 >= 0) step3(f - 2, x2, x1);
    if (f - 3 >= 0) step3(f - 3, x3, x2);
    if (f - 4 >= 0) step3(f - 4, x4, x3);
  }
}

}  // namespace wg
