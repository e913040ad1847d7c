// Column kernel of one acoustic substep, level-parallel version.
//
// A block owns TX (16 or 32) adjacent columns of one row j and all levels.
// Its TY level lanes split the levels (lane l handles k = l, l+TY, ...) for
// every part of advance_mu_t / advance_w / calc_p_rho that is independent
// across levels; only the four genuine column recurrences run serially, one
// thread per column, out of shared memory:
//   * dmdt = sum_k dnw*dvdxi            (dynamics/mu_t_advance.py:205)
//   * the ww prefix subtraction         (dynamics/mu_t_advance.py:229-237)
//   * the Thomas forward and back sweeps (core/advance_w.py:558-592)
// Every expression keeps the operation order of the thread-per-column form
// (and of the reference), so results are identical to it bit for bit.
#pragma once
#include "dycore_common.cuh"
#include "acoustic_kernels.cuh"

namespace wg {

// Block shape: TX columns x TY level lanes (template parameters, tuned per
// grid; COL_TX x COL_TY is the default); col_minb(TX) resident blocks per SM
// requested from the register allocator.
#ifndef WG_COL_TX
#define WG_COL_TX 32
#endif
#ifndef WG_COL_TY
#define WG_COL_TY 17
#endif
#ifndef WG_COL_MINB
#define WG_COL_MINB 2
#endif
// L2 prefetch of the block's input rows: 0 off, 1 all at block start, 2 in
// two groups (advance_mu_t inputs at start, advance_w inputs after P4).
#ifndef WG_COL_PREFETCH
#define WG_COL_PREFETCH 2
#endif
constexpr int COL_TX = WG_COL_TX;
constexpr int COL_TY = WG_COL_TY;
constexpr int COL_NARR = 8;
// Column widths and level-lane counts the column kernel is instantiated for
// (the tuner's choices).  A 16-column block holds half the shared memory of a
// 32-column one, so twice as many blocks are resident per SM.
constexpr int COL_TX_CHOICES[] = {32, 16, 1};
// Width of the default column kernel: 1 selects the one-thread-per-column
// streaming kernel (column_stream.cuh), 16 or 32 this level-parallel one.
#ifndef WG_COL_DEFAULT_WIDTH
#define WG_COL_DEFAULT_WIDTH 32
#endif
constexpr int COL_DEFAULT_WIDTH = WG_COL_DEFAULT_WIDTH;
constexpr int COL_TY_CHOICES[] = {8, 13, 16, 17};
constexpr int col_minb(int tx) { return tx == 16 ? 2 * WG_COL_MINB : WG_COL_MINB; }
// Levels per software-pipelined batch of the serial recurrences: the batch's
// shared-memory operands are loaded before its first store, so the loads
// overlap instead of each waiting behind the previous level's store.
#ifndef WG_COL_SU
#define WG_COL_SU 8
#endif
constexpr int COL_SU = WG_COL_SU;

// Bulk L2 prefetch of the rows (levels 0..nz) this column block will read.
// group 0: advance_mu_t / theta / t_2ave inputs; group 1: advance_w and
// calc_p_rho inputs.  (u_1 and v_1 are read at levels 0..2 only, for the
// surface w, and are not prefetched.)
template <int TX>
__device__ __forceinline__ void column_prefetch(const Grid &g, const Acoustic &A, const ColArgs &c,
                                                const double *hdiv, int group, int i0, int j) {
  const int nx = g.nx, ny = g.ny, nz = g.nz, L = nz + 1;
  const int w = min(TX, nx - i0);
  constexpr int nrows = 10;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int e = tid; e < nrows * L; e += blockDim.x * blockDim.y) {
    const int r = e / L, k = e - r * L;
    const double *p = nullptr;
    const bool mass = k < nz;
    if (group == 0) {
      switch (r) {
        case 0: p = A.ww_1 + ix3(k, j, i0, ny, nx); break;
        case 1: p = A.ww + ix3(k, j, i0, ny, nx); break;
        case 2: if (mass) p = A.theta_w + ix3(k, j, i0, ny, nx); break;
        case 3: if (mass) p = A.t2ave + ix3(k, j, i0, ny, nx); break;
        case 4: if (mass) p = A.t_tend + ix3(k, j, i0, ny, nx); break;
        case 5: if (mass) p = A.theta_s + ix3(k, j, i0, ny, nx); break;
        case 6: if (mass) p = A.c2a + ix3(k, j, i0, ny, nx); break;
        case 7: if (mass) p = A.alt + ix3(k, j, i0, ny, nx); break;
        case 8: if (mass) p = hdiv + ix3(k, j, i0, ny, nx); break;
        default: p = A.pt1 + ix3(k, j, i0, ny, nx); break;
      }
    } else {
      switch (r) {
        case 0: p = A.ph + ix3(k, j, i0, ny, nx); break;
        case 1: p = A.ph_tend + ix3(k, j, i0, ny, nx); break;
        case 2: p = A.w + ix3(k, j, i0, ny, nx); break;
        case 3: p = A.rw_tend + ix3(k, j, i0, ny, nx); break;
        case 4: p = A.cqw + ix3(k, j, i0, ny, nx); break;
        case 5: p = A.a + ix3(k, j, i0, ny, nx); break;
        case 6: p = A.alpha + ix3(k, j, i0, ny, nx); break;
        case 7: p = A.gamma + ix3(k, j, i0, ny, nx); break;
        case 8: if (c.damp_opt == 3) p = A.w_save + ix3(k, j, i0, ny, nx); break;
        default: if (mass) p = A.pm1 + ix3(k, j, i0, ny, nx); break;
      }
    }
    if (p != nullptr) l2_prefetch_row(p, w);
  }
}

inline size_t column_tiled_smem_bytes(int nz, int tx) { return (size_t)COL_NARR * (nz + 1) * tx * sizeof(double); }

// PIN: compile in the boundary cadence's ring-0 pins of mu / muts / muave and
// the work theta, and the ring-0 ph pin (cadence and nested child); off, the
// kernel carries no trace of them.
template <int TX, int TY, bool PIN = false>
__global__ void __launch_bounds__(TX * TY, col_minb(TX)) k_column_tiled(Grid g, Acoustic A, ColArgs c,
                                                                         const double *dvdxi, const double *hdiv) {
  static_assert(TX == 16 || TX == 32, "a column block is 16 or 32 columns wide");
  // rows ty < R0 share warp 0 with the serial thread row ty == 0
  constexpr int R0 = 32 / TX;
  static_assert(TY > R0, "the Thomas phase needs a warp besides warp 0 to stage gamma");
  extern __shared__ double sm[];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = blockIdx.x * TX + tx;
  const int j = blockIdx.y;
  const bool valid = i < nx;
  const int L = nz + 1;
  auto S = [&](int a, int k) -> double & { return sm[((size_t)a * L + k) * TX + tx]; };
  // array roles (see the phase list below)
  constexpr int A0 = 0, A1 = 1, A2 = 2, A3 = 3, A4 = 4, A5 = 5, A6 = 6, A7 = 7;
  const size_t c2d = valid ? ix2(j, i, nx) : 0;
  auto M = [&](int k) { return ix3(k, j, i, ny, nx); };
  const double dts = c.dts;
  const double eps_p = 1.0 + c.epssm, eps_m = 1.0 - c.epssm;
  const double msftx = valid ? ld(g.msftx, c2d) : 1.0;
  const double msfty = valid ? ld(g.msfty, c2d) : 1.0;
  const double mut = valid ? ld(A.mut, c2d) : 1.0;
  const double minv = valid ? ld(g.rmsfty, c2d) : 1.0;  // == 1.0 / msfty
  const bool active = valid && (!c.specified || (j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2));
  auto T1 = [&](int k, int jj, int ii2) { return ld(A.theta_s, ix3(k, jj, ii2, ny, nx)) - T0; };
  const int nxu = nx + 1, nyv = ny + 1;

  __shared__ double s_dmdt[TX], s_mutend[TX], s_scale[TX];
  // 2-D inputs of the serial phases, loaded early so their latency overlaps P1
  double muts_in = 0.0, mu_in = 0.0, mu_tend_in = 0.0;
  if (ty == 0 && active) {
    muts_in = A.muts[c2d];
    mu_in = A.mu[c2d];
    mu_tend_in = (A.mu_tend != nullptr) ? ld(A.mu_tend, c2d) : 0.0;
  }
  if (WG_COL_PREFETCH >= 1) column_prefetch<TX>(g, A, c, hdiv, 0, blockIdx.x * TX, j);
  if (WG_COL_PREFETCH == 1) column_prefetch<TX>(g, A, c, hdiv, 1, blockIdx.x * TX, j);

  // ---------------- P1: dvdxi per level (from k_div_h) -> A0 ----------------
  if (active) {
    for (int k = ty; k < nz; k += TY) S(A0, k) = ld(dvdxi, M(k));
  }
  __syncthreads();
  // ---------------- P2: column sum and 2-D mass updates (serial, ty == 0) ----------------
  if (ty == 0 && active) {
    double dmdt = 0.0;
    int k = 0;
    for (; k + COL_SU <= nz; k += COL_SU) {
      double t[COL_SU];
#pragma unroll
      for (int u = 0; u < COL_SU; ++u) t[u] = ld(g.dnw, k + u) * S(A0, k + u);
#pragma unroll
      for (int u = 0; u < COL_SU; ++u) dmdt = (k + u == 0) ? t[u] : dmdt + t[u];
    }
    for (; k < nz; ++k) {
      const double t = ld(g.dnw, k) * S(A0, k);
      dmdt = (k == 0) ? t : dmdt + t;
    }
    const double mu_work_old = muts_in - mut;
    const double mu_save = mu_in - mu_work_old;
    double mu_tend = mu_tend_in;
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
    s_dmdt[tx] = dmdt;
    s_mutend[tx] = mu_tend;
    s_scale[tx] = scale;
  }
  if (PIN && ty == 0 && valid && !active && c.cad) {
    // specified cadence: ring-0 mu', muts and muave pinned to the mu' leaf
    const double mu_pin = ring_target(c.cad_mu, 1, ny, nx, 0, j, i);
    const double muts_pin = ld(c.mub, c2d) + mu_pin;
    A.mu[c2d] = mu_pin;
    A.muts[c2d] = muts_pin;
    A.muave[c2d] = muts_pin - mut;
  }
  __syncthreads();
  // ---------------- P3: ww increments -> A1, ww_1 -> A2, old ww (inactive) -> A3 ----------------
  // P5's per-level inputs are copied asynchronously now, each level by the
  // thread that will use it: theta_w -> A7 (kept to P10), old t_2ave -> A6
  // and t_tend -> A4 (both free until P6/P7).
  if (valid) {
    for (int k = ty; k < nz; k += TY) {
      cp_async8(&S(A7, k), A.theta_w + M(k));
      cp_async8(&S(A6, k), A.t2ave + M(k));
      cp_async8(&S(A4, k), A.t_tend + M(k));
    }
  }
  cp_async_commit();
  double ww_bot = 0.0, ww_top = 0.0;  // old ww at faces 0 and nz, for P4
  if (ty == 0 && active) {
    ww_bot = A.ww[M(0)];
    ww_top = A.ww[M(nz)];
  }
  if (valid) {
    if (active) {
      const double dmdt = s_dmdt[tx], mu_tend = s_mutend[tx], scale = s_scale[tx];
      for (int kk = 1 + ty; kk < nz; kk += TY) {
        const int k = kk - 1;
        double dv = S(A0, k);
        if (c.specified) dv = dv * scale;
        S(A1, kk) = div_rcp(ld(g.dnw, k) * (ld(g.c1h, k) * dmdt + dv + ld(g.c1h, k) * mu_tend), msfty, minv);
      }
      for (int k = ty; k <= nz; k += TY) S(A2, k) = ld(A.ww_1, M(k));
    } else {
      for (int k = ty; k <= nz; k += TY) S(A3, k) = A.ww[M(k)];
    }
  }
  __syncthreads();
  // ---------------- P4: ww prefix (serial) -> A3 ----------------
  if (ty == 0 && active) {
    double prev = ww_bot;
    S(A3, 0) = prev - S(A2, 0);
    int kk = 1;
    for (; kk + COL_SU <= nz; kk += COL_SU) {
      double r1[COL_SU], r2[COL_SU];
#pragma unroll
      for (int u = 0; u < COL_SU; ++u) {
        r1[u] = S(A1, kk + u);
        r2[u] = S(A2, kk + u);
      }
#pragma unroll
      for (int u = 0; u < COL_SU; ++u) {
        const double cur = prev - r1[u];
        S(A3, kk + u) = cur - r2[u];
        prev = cur;
      }
    }
    for (; kk < nz; ++kk) {
      const double cur = prev - S(A1, kk);
      S(A3, kk) = cur - S(A2, kk);
      prev = cur;
    }
    S(A3, nz) = ww_top;
  }
  __syncthreads();
  if (WG_COL_PREFETCH == 2) column_prefetch<TX>(g, A, c, hdiv, 1, blockIdx.x * TX, j);
  // ---------------- P5: theta update, t_2ave, wd -> A0, buoy -> A1, coef -> A5 ----------------
  const double muts = valid ? A.muts[c2d] : 1.0;
  const double muave = valid ? A.muave[c2d] : 0.0;
  if (valid) {
    for (int k = ty; k <= nz; k += TY) A.ww[M(k)] = S(A3, k);
    cp_async_wait<0>();  // this thread's staged levels
    for (int k = ty; k < nz; k += TY) {
      double thw = S(A7, k);
      const double t2ave_old = S(A6, k);
      if (active) {
        const double wdtn_hi = (k + 1 <= nz - 1)
                                   ? S(A3, k + 1) * (ld(g.fnm, k + 1) * T1(k + 1, j, i) + ld(g.fnp, k + 1) * T1(k, j, i))
                                   : 0.0;
        const double wdtn_lo = (k >= 1) ? S(A3, k) * (ld(g.fnm, k) * T1(k, j, i) + ld(g.fnp, k) * T1(k - 1, j, i)) : 0.0;
        // horizontal theta flux divergence from k_div_h (same expression)
        const double tend = ld(hdiv, M(k)) + ld(g.rdnw, k) * (wdtn_hi - wdtn_lo);
        const double theta_i = thw + msfty * dts * S(A4, k);
        thw = theta_i - dts * msfty * tend;
        A.theta_w[M(k)] = thw;
        S(A7, k) = thw;
      } else if (PIN && c.cad) {
        // specified cadence: the ring-0 work theta whose finished theta is the leaf's
        const double mass_pin = ld(g.c1h, k) * muts + ld(g.c2h, k);
        const double mass_cur = ld(g.c1h, k) * mut + ld(g.c2h, k);
        thw = mass_pin * (ring_target(c.cad_th, nz, ny, nx, k, j, i) - T0) - mass_cur * T1(k, j, i);
        A.theta_w[M(k)] = thw;
        S(A7, k) = thw;
      }
      const double mass_h = ld(g.c1h, k) * muts + ld(g.c2h, k);
      const double half = 0.5 * (eps_p * thw + eps_m * t2ave_old);
      const double t2a = (half + (ld(g.c1h, k) * muave) * T0) / (mass_h * (T0 + T1(k, j, i)));
      A.t2ave[M(k)] = t2a;
      const double c2a_k = ld(A.c2a, M(k));
      S(A1, k) = c2a_k * ld(A.alt, M(k)) * t2a;
      S(A5, k) = c2a_k * ld(g.rdnw, k) / safe12(ld(g.c1h, k) * mut + ld(g.c2h, k));  // coef(k) for P7
      const double wwm = 0.5 * (S(A3, k + 1) + S(A3, k));
      S(A0, k) = wwm * ld(g.rdnw, k) * (ld(A.pt1, M(k + 1)) - ld(A.pt1, M(k)));
    }
  }
  __syncthreads();
  // ---------------- P6: rhs -> A2 (faces 1..nz), old ph -> A4 (faces 0..nz) ----------------
  const double c05gem = 0.5 * G * eps_m;
  if (valid) {
    for (int f = ty; f <= nz; f += TY) {
      const double phf = ld(A.ph, M(f));
      S(A4, f) = phf;
      if (f == 0) {
        S(A2, 0) = 0.0;
        continue;
      }
      double r = dts * (ld(A.ph_tend, M(f)) + c05gem * ld(A.w, M(f)));
      if (f < nz) r = r + (-(dts * (ld(g.fnm, f) * S(A0, f) + ld(g.fnp, f) * S(A0, f - 1))));
      const double mf = ld(g.c1f, f) * mut + ld(g.c2f, f);
      r = phf + msfty * r / mf;
      if (f == nz && c.top_lid) r = 0.0;
      S(A2, f) = r;
    }
  }
  __syncthreads();
  // ---------------- P7: explicit w -> A6 (coef from A5); then a -> A0, alpha -> A3, gamma -> A5 ----------------
  if (valid) {
    const double c05dg = 0.5 * dts * G;
    const double dtsg = dts * G;
    for (int f = ty; f <= nz; f += TY) {
      const double a_f = ld(A.a, M(f)), alpha_f = ld(A.alpha, M(f));
      double wn;
      if (f == 0) {
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
        wn = msfty * 0.5 * g.rdy * (dy_n * vcf(j + 1) + dy_s * vcf(j)) +
             msftx * 0.5 * g.rdx * (dx_e * ucf(i + 1) + dx_w * ucf(i));
      } else if (f < nz) {
        const double w_old = ld(A.w, M(f));
        double rw = ld(A.rw_tend, M(f));
        if (c.w_damping == 1) {
          const double mf = ld(g.c1f, f) * mut + ld(g.c2f, f);
          const double vert_cfl = fabs(S(A3, f) / safe12(mf) * ld(g.rdnw, f) * dts);
          double damp = -sgn(w_old) * W_ALPHA * (vert_cfl - W_BETA) * mf;
          damp = (vert_cfl > W_BETA) ? damp : 0.0;
          rw = rw + damp;
        }
        wn = w_old + dts * rw;
        const double coef_f = S(A5, f), coef_m1 = S(A5, f - 1);
        const double tA_u = coef_f * (eps_p * (S(A2, f + 1) - S(A2, f)) + eps_m * (S(A4, f + 1) - S(A4, f)));
        const double tA_l = coef_m1 * (eps_p * (S(A2, f) - S(A2, f - 1)) + eps_m * (S(A4, f) - S(A4, f - 1)));
        const double tA = minv * ld(A.cqw, M(f)) * (c05dg * ld(g.rdn, f)) * (tA_u - tA_l);
        const double tB = dtsg * minv * (ld(g.rdn, f) * (S(A1, f) - S(A1, f - 1)) - (ld(g.c1f, f) * muave));
        wn = wn + (tA + tB);
      } else {
        const int km1 = nz - 1;
        const double mhm = safe12(ld(g.c1h, km1) * mut + ld(g.c2h, km1));
        const double rdnw_t = ld(g.rdnw, km1);
        const double t2a_t = A.t2ave[M(km1)];
        const double tA_top = -0.5 * dts * G / mhm * (rdnw_t * rdnw_t) * 2.0 * ld(A.c2a, M(km1)) *
                              (eps_p * (S(A2, nz) - S(A2, nz - 1)) + eps_m * (S(A4, nz) - S(A4, nz - 1)));
        const double tB_top = -dts * G * (2.0 * rdnw_t * ld(A.c2a, M(km1)) * ld(A.alt, M(km1)) * t2a_t + (ld(g.c1f, nz) * muave));
        const double w_top = ld(A.w, M(nz)) + dts * ld(A.rw_tend, M(nz)) + minv * (tA_top + tB_top);
        wn = c.top_lid ? 0.0 : w_top;
      }
      S(A6, f) = wn;
      S(A0, f) = a_f;      // wd(f) was last read in P6
      S(A3, f) = alpha_f;  // ww(f) was last read above, by this thread
    }
  }
  __syncthreads();
  // ---------------- P8: Thomas forward (serial) while the other warps stage gamma -> A5 ----------------
  if (ty == 0) {
    if (valid) {
      double wf_prev = S(A6, 0);
      int f = 1;
      for (; f + COL_SU - 1 <= nz; f += COL_SU) {
        double r6[COL_SU], r0[COL_SU], r3[COL_SU];
#pragma unroll
        for (int u = 0; u < COL_SU; ++u) {
          r6[u] = S(A6, f + u);
          r0[u] = S(A0, f + u);
          r3[u] = S(A3, f + u);
        }
#pragma unroll
        for (int u = 0; u < COL_SU; ++u) {
          const double wf = (r6[u] - r0[u] * wf_prev) * r3[u];
          S(A6, f + u) = wf;
          wf_prev = wf;
        }
      }
      for (; f <= nz; ++f) {
        const double wf = (S(A6, f) - S(A0, f) * wf_prev) * S(A3, f);
        S(A6, f) = wf;
        wf_prev = wf;
      }
    }
  } else if (ty >= R0 && valid) {
    for (int f = ty - R0; f <= nz; f += TY - R0) S(A5, f) = ld(A.gamma, M(f));
  }
  __syncthreads();
  // ---------------- P8b: Thomas back substitution (serial) ----------------
  if (ty == 0 && valid) {
    double ws_next = S(A6, nz);
    int f = nz - 1;
    for (; f - COL_SU + 1 >= 1; f -= COL_SU) {
      double r6[COL_SU], r5[COL_SU];
#pragma unroll
      for (int u = 0; u < COL_SU; ++u) {
        r6[u] = S(A6, f - u);
        r5[u] = S(A5, f - u);
      }
#pragma unroll
      for (int u = 0; u < COL_SU; ++u) {
        const double ws = r6[u] - r5[u] * ws_next;
        S(A6, f - u) = ws;
        ws_next = ws;
      }
    }
    for (; f >= 1; --f) {
      const double ws = S(A6, f) - S(A5, f) * ws_next;
      S(A6, f) = ws;
      ws_next = ws;
    }
  }
  __syncthreads();
  // ---------------- P9: Rayleigh damping, w out, phi finish -> A4 ----------------
  if (valid) {
    const bool do_damp = (c.damp_opt == 3 && c.dampcoef > 0.0);
    double dampmag = 0.0, hbot = 0.0;
    if (do_damp) {
      dampmag = dts * c.dampcoef;
      hbot = div_rcp(ld(A.pt1, M(nz)), G, RG) - c.zdamp;
    }
    for (int f = ty; f <= nz; f += TY) {
      double ws = S(A6, f);
      if (f >= 1) {
        if (do_damp) {
          const double hk = div_rcp(ld(A.pt1, M(f)), G, RG);
          const double sv = sin(over_zdamp(0.5 * 3.141592653589793 * (hk - hbot), c));
          const double ramp = sv * sv;
          const double dampwt = (hk >= hbot) ? dampmag * ramp : 0.0;
          const double mf = ld(g.c1f, f) * mut + ld(g.c2f, f);
          ws = (ws - dampwt * mf * ld(A.w_save, M(f))) / (1.0 + dampwt);
        }
        const double mfs = ld(g.c1f, f) * muts + ld(g.c2f, f);
        const double phn = S(A2, f) + msfty * 0.5 * dts * G * eps_p * ws / mfs;
        S(A4, f) = phn;
        A.ph[M(f)] = phn;
      }
      if (PIN && !active && c.ph_pin) {
        // ring-0 work ph whose finished ph' is the leaf's (spec_bdyupdate_ph)
        const double phn = ring_target(c.cad_ph, nz + 1, ny, nx, f, j, i) - ld(c.ph_save, M(f));
        S(A4, f) = phn;
        A.ph[M(f)] = phn;
      }
      A.w[M(f)] = ws;
    }
  }
  __syncthreads();
  // ---------------- P10: calc_p_rho with smdiv memory ----------------
  if (valid) {
    const double mu_work = muts - mut;
    for (int k = ty; k < nz; k += TY) {
      const double mass = ld(g.c1h, k) * muts + ld(g.c2h, k);
      const double safe = safe12(mass);
      const double mu_term = ld(g.c1h, k) * mu_work;
      const double altc = ld(A.alt, M(k));
      const double al = -(altc * mu_term + ld(g.rdnw, k) * (S(A4, k + 1) - S(A4, k))) / safe;
      const double t1 = T1(k, j, i);
      const double ttr = T0 + t1;
      const double sttr = fabs(ttr) > 1.0e-6 ? ttr : 1.0e-6;
      const double pp = ld(A.c2a, M(k)) * (altc * (S(A7, k) - mu_term * t1) / (safe * sttr) - al);
      const double pm1 = ld(A.pm1, M(k));
      A.p[M(k)] = pp + SMDIV * (pp - pm1);
      A.pm1[M(k)] = pp;
      A.al[M(k)] = al;
    }
  }
}

}  // namespace wg
