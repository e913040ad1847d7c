// Flux-form scalar advection operator (h5/v3, periodic) and its hand-written
// adjoints with respect to the advected field and the transport velocities.
//
// For fixed transport velocities (ru, rv at the cells' west / south faces,
// rom at the w faces) the tendency tend = L(ru, rv, rom) q of
// flux_advection.py:482-568 is linear in q: the upwind switch sign(vel)
// depends on the velocity only.  k_scalar_adv_op applies L; k_scalar_adv_vjp
// applies its transpose L^T to a tendency-space vector lambda (and forms the
// velocities' cotangents, below):
//
//   face flux   F_f = vel_f * sum_m w_m(sign vel_f) q(stencil_f, m)
//   tendency    tend(c) = -msftx rdx (Fx(c+1) - Fx(c)) - msftx rdy (Fy(c+1) - Fy(c))
//                          - rdnw(k) (Fz(k+1) - Fz(k))
//   adjoint     Fbar_f = d tend / d F_f . lambda   (two cells per face)
//               qbar(c) = sum over the faces whose stencil holds c of
//                         vel_f w_m(sign vel_f) Fbar_f
//
// gathered per cell (no atomics).  The flux5 weights follow from
// (37(q0+q-1) - 8(q+1+q-2) + (q+2+q-3))/60 - s((q+2-q-3) - 5(q+1-q-2) + 10(q0-q-1))/60,
// the flux3 weights from (7(q0+q-1) - (q+1+q-2))/12 + s'((q+1-q-2) - 3(q0-q-1))/12
// with s' = sign(-vel) (flux_advection.py:53-88, 534-562).
#pragma once
#include "dycore_common.cuh"
#include "stage_kernels.cuh"
#include "tiled_stencils.cuh"

namespace wg {

struct AdvOpArgs {
  const double *ru, *rv, *rom;  // (nz, ny, nx), (nz, ny, nx), (nz+1, ny, nx)
  // (ny, nx) factors of the horizontal and the vertical flux divergence: the
  // scalar's msftx and 1 (vfac NULL); msfux and 1 for u's core faces;
  // msfvy and msfvy / msfvx for v's (flux_advection.py:1131-1274)
  const double *hfac, *vfac;
};

__global__ void k_scalar_adv_op(Grid g, AdvOpArgs v, const double *q, double *tend) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  auto Q = [&](int kk, int jj, int ii) { return ld(q, ix3(kk, wrp(jj, ny), wrp(ii, nx), ny, nx)); };
  auto fx = [&](int ii) {  // flux at the west face of cell (k, j, ii)
    const double vel = ld(v.ru, ix3(k, j, wrp(ii, nx), ny, nx));
    return hflux5<double>(vel, Q(k, j, ii - 3), Q(k, j, ii - 2), Q(k, j, ii - 1), Q(k, j, ii), Q(k, j, ii + 1),
                          Q(k, j, ii + 2));
  };
  auto fy = [&](int jj) {
    const double vel = ld(v.rv, ix3(k, wrp(jj, ny), i, ny, nx));
    return hflux5<double>(vel, Q(k, jj - 3, i), Q(k, jj - 2, i), Q(k, jj - 1, i), Q(k, jj, i), Q(k, jj + 1, i),
                          Q(k, jj + 2, i));
  };
  const double hf = ld(v.hfac, ix2(j, i, nx));
  double t = -hf * g.rdx * (fx(i + 1) - fx(i));
  t = t - hf * g.rdy * (fy(j + 1) - fy(j));
  if (v.rom == nullptr) {  // the horizontal flux divergence alone
    tend[ix3(k, j, i, ny, nx)] = t;
    return;
  }
  auto qc = [&](int kk) { return ld(q, ix3(kk, j, i, ny, nx)); };
  const double v1 = (k + 1 <= nz - 1) ? vflux3_at(g, k + 1, ld(v.rom, ix3(k + 1, j, i, ny, nx)), qc) : 0.0;
  const double v0 = (k >= 1) ? vflux3_at(g, k, ld(v.rom, ix3(k, j, i, ny, nx)), qc) : 0.0;
  if (v.vfac == nullptr)
    tend[ix3(k, j, i, ny, nx)] = t - ld(g.rdnw, k) * (v1 - v0);
  else
    tend[ix3(k, j, i, ny, nx)] = t + ld(v.vfac, ix2(j, i, nx)) * (-(ld(g.rdnw, k) * (v1 - v0)));
}

// flux5 weight of stencil position m (0..5 = q-3..q+2) for upwind sign s,
// and the flux3 weight of position m (0..3 = q(m-2)..q(m+1)) for
// s' = sign(-vel).  s takes the values -1, 0, 1 only, so every weight is one
// of three constants folded at compile time (the same quotients a runtime
// division gives); the loops that call these unroll m.
__host__ __device__ constexpr double w5c(int m, double s) {
  return m == 0 ? (1.0 + s) / 60.0
       : m == 1 ? (-8.0 - 5.0 * s) / 60.0
       : m == 2 ? (37.0 + 10.0 * s) / 60.0
       : m == 3 ? (37.0 - 10.0 * s) / 60.0
       : m == 4 ? (-8.0 + 5.0 * s) / 60.0
                : (1.0 - s) / 60.0;
}
__host__ __device__ constexpr double w3c(int m, double s) {
  return m == 0 ? (-1.0 - s) / 12.0 : m == 1 ? (7.0 + 3.0 * s) / 12.0 : m == 2 ? (7.0 - 3.0 * s) / 12.0 : (-1.0 + s) / 12.0;
}
template <int M>
__device__ __forceinline__ double w5(double s) {
  constexpr double p = w5c(M, 1.0), z = w5c(M, 0.0), n = w5c(M, -1.0);
  return s > 0.0 ? p : (s < 0.0 ? n : z);
}
__device__ __forceinline__ double w5(int m, double s) {
  switch (m) {
    case 0: return w5<0>(s);
    case 1: return w5<1>(s);
    case 2: return w5<2>(s);
    case 3: return w5<3>(s);
    case 4: return w5<4>(s);
    default: return w5<5>(s);
  }
}
template <int M>
__device__ __forceinline__ double w3(double s) {
  constexpr double p = w3c(M, 1.0), z = w3c(M, 0.0), n = w3c(M, -1.0);
  return s > 0.0 ? p : (s < 0.0 ? n : z);
}
__device__ __forceinline__ double w3(int m, double s) {
  switch (m) {
    case 0: return w3<0>(s);
    case 1: return w3<1>(s);
    case 2: return w3<2>(s);
    default: return w3<3>(s);
  }
}

// The full vector-Jacobian product.  tend is bilinear in (q, vel): with the
// upwind signs frozen each face flux is F_f = vel_f h_f(q), so
//   Fbar_x(i) = rdx (hfac(i) lam(i) - hfac(i-1) lam(i-1)), likewise y,
//   Fbar_z(m) = vfac (rdnw(m) lam(m) - rdnw(m-1) lam(m-1)),
//   q_bar(c)  = sum over the faces whose stencil holds c of
//               vel_f w_m(sign vel_f) Fbar_f            (a gather, no atomics)
//   velbar_f  = Fbar_f h_f(q),   h_f = flux5 / flux3 of the face's stencil
//               (the second-order face value at m = 1 and nz-1).
// One 32 x 8 block per tile and level: the level's hfac*lam, ru, rv (and,
// for the velocity cotangents, q) plane tiles are staged in shared memory
// with their periodic halos, the vertical stencils read the column.  q_bar,
// ru_bar, rv_bar at cell (k, j, i) and its west / south face for k < nz,
// rom_bar at w face (k, j, i) (zero at k = 0 and nz, whose fluxes are zero).
// Outputs given as NULL are skipped.
__global__ void __launch_bounds__(TSX * TSY) k_scalar_adv_vjp(Grid g, AdvOpArgs v, const double *q,
                                                               const double *lam, double *q_bar, double *ru_bar,
                                                               double *rv_bar, double *rom_bar) {
  using TM = Tile<3, 3>;  // hfac * lam
  using TU = Tile<3, 0>;  // ru: west faces of cells i0-3 .. i0+34
  using TV = Tile<0, 3>;  // rv: south faces of rows j0-3 .. j0+10
  __shared__ double sml[TM::N], sru[TU::N], srv[TV::N], sq[TM::N];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * TSX, j0 = blockIdx.y * TSY, k = blockIdx.z;
  const int i = i0 + tx, j = j0 + ty;
  const bool valid = i < nx && j < ny;
  if (k < nz) {
    const size_t kp = (size_t)k * ny * nx;
    for (int e = ty * TSX + tx; e < TM::N; e += TSX * TSY) {
      const int r = e / TM::W, c = e - r * TM::W;
      const int jj = wrp(j0 - 3 + r, ny), ii = wrp(i0 - 3 + c, nx);
      sml[e] = ld(v.hfac, ix2(jj, ii, nx)) * ld(lam, kp + ix2(jj, ii, nx));
    }
    load_tile<3, 0>(sru, v.ru + kp, nx, i0, j0, nx, ny, 0.0);
    load_tile<0, 3>(srv, v.rv + kp, nx, i0, j0, nx, ny, 0.0);
    if (ru_bar != nullptr || rv_bar != nullptr) load_tile<3, 3>(sq, q + kp, nx, i0, j0, nx, ny, 0.0);
    __syncthreads();
    if (valid) {
      auto ML = [&](int r, int cc) { return sml[(r + 3) * TM::W + (cc + 3)]; };
      auto RU = [&](int cc) { return sru[ty * TU::W + (cc + 3)]; };
      auto RV = [&](int r) { return srv[(r + 3) * TV::W + tx]; };
      auto Q = [&](int r, int cc) { return sq[(r + 3) * TM::W + (cc + 3)]; };
      double acc = 0.0;
      // x faces of cells i-2 .. i+3 whose stencils hold this cell (position 3 - t)
#pragma unroll
      for (int t = -2; t <= 3; ++t) {
        const double vel = RU(tx + t);
        acc += vel * w5(3 - t, sgn(vel)) * (g.rdx * (ML(ty, tx + t) - ML(ty, tx + t - 1)));
      }
      if (ru_bar != nullptr)
        ru_bar[kp + ix2(j, i, nx)] = g.rdx * (ML(ty, tx) - ML(ty, tx - 1)) *
                                     flux5(Q(ty, tx - 3), Q(ty, tx - 2), Q(ty, tx - 1), Q(ty, tx), Q(ty, tx + 1),
                                           Q(ty, tx + 2), RU(tx));
#pragma unroll
      for (int t = -2; t <= 3; ++t) {
        const double vel = RV(ty + t);
        acc += vel * w5(3 - t, sgn(vel)) * (g.rdy * (ML(ty + t, tx) - ML(ty + t - 1, tx)));
      }
      if (rv_bar != nullptr)
        rv_bar[kp + ix2(j, i, nx)] = g.rdy * (ML(ty, tx) - ML(ty - 1, tx)) *
                                     flux5(Q(ty - 3, tx), Q(ty - 2, tx), Q(ty - 1, tx), Q(ty, tx), Q(ty + 1, tx),
                                           Q(ty + 2, tx), RV(ty));
      if (q_bar != nullptr && v.rom == nullptr) q_bar[kp + ix2(j, i, nx)] = acc;
      if (q_bar != nullptr && v.rom != nullptr) {
        // z faces m = k-1 .. k+2 whose stencils hold level k
        const double vf = v.vfac != nullptr ? ld(v.vfac, ix2(j, i, nx)) : 1.0;
        auto Lz = [&](int kk) { return vf * ld(lam, ix3(kk, j, i, ny, nx)); };
#pragma unroll
        for (int t = -1; t <= 2; ++t) {
          const int m = k + t;
          if (m < 1 || m > nz - 1) continue;
          const double rom = ld(v.rom, ix3(m, j, i, ny, nx));
          double wk = 0.0;
          if (m == 1 || m == nz - 1) {
            if (t == 0) wk = ld(g.fnm, m);
            else if (t == 1) wk = ld(g.fnp, m);
          } else {
            wk = w3(2 - t, sgn(-rom));  // stencil q(m-2) .. q(m+1): level k is position 2 - t
          }
          acc += rom * wk * (ld(g.rdnw, m) * Lz(m) - ld(g.rdnw, m - 1) * Lz(m - 1));
        }
        q_bar[kp + ix2(j, i, nx)] = acc;
      }
    }
  }
  if (rom_bar != nullptr && v.rom != nullptr && valid) {
    double r = 0.0;
    if (k >= 1 && k <= nz - 1) {
      auto qc = [&](int kk) { return ld(q, ix3(kk, j, i, ny, nx)); };
      const double vf = v.vfac != nullptr ? ld(v.vfac, ix2(j, i, nx)) : 1.0;
      auto L = [&](int kk) { return vf * ld(lam, ix3(kk, j, i, ny, nx)); };
      const double rom = ld(v.rom, ix3(k, j, i, ny, nx));
      double h;
      if (k == 1 || k == nz - 1) {
        h = ld(g.fnm, k) * qc(k) + ld(g.fnp, k) * qc(k - 1);
      } else {
        const double s = sgn(-rom);
        h = w3(0, s) * qc(k - 2) + w3(1, s) * qc(k - 1) + w3(2, s) * qc(k) + w3(3, s) * qc(k + 1);
      }
      r = (ld(g.rdnw, k) * L(k) - ld(g.rdnw, k - 1) * L(k - 1)) * h;
    }
    rom_bar[ix3(k, j, i, ny, nx)] = r;
  }
}

// ---------------------------------------------------------------------------
// The vertical flux divergence of w (flux_advection.py:1410-1482, the
// oracle's _vdiv_w) on its nz+1 levels: vel(k) = (rom(k) + rom(k-1)) / 2,
// face values flux3 with the -sign(vel) correction for k = 2..nz-1 and
// (w(k) + w(k-1)) / 2 at k = 1 and, without a rigid lid, at k = nz;
// tend(k) = -rdn(k) (vflux(k+1) - vflux(k)) for k = 1..nz-1 and, without a
// lid, tend(nz) = 2 rdn(nz-1) vflux(nz).  Index space (nx, ny, nz+1).
// ---------------------------------------------------------------------------
struct WColumn {
  const double *w, *rom;  // (nz+1, ny, nx) each
  int top_lid;
};

__device__ __forceinline__ double wvel(const Grid &g, const WColumn &c, int k, int j, int i) {
  return 0.5 * (ld(c.rom, ix3(k, j, i, g.ny, g.nx)) + ld(c.rom, ix3(k - 1, j, i, g.ny, g.nx)));
}
// vflux(k) / vel(k): the face value of w at w-level face k (0 where there is no flux)
__device__ __forceinline__ double wface(const Grid &g, const WColumn &c, int k, int j, int i, double vel) {
  const int nz = g.nz;
  auto W = [&](int kk) { return ld(c.w, ix3(kk, j, i, g.ny, g.nx)); };
  if (k == 1) return 0.5 * (W(1) + W(0));
  if (k >= 2 && k <= nz - 1) {
    const double flux4 = div_rcp(7.0 * (W(k) + W(k - 1)) - (W(k + 1) + W(k - 2)), 12.0, R12);
    const double corr = div_rcp((W(k + 1) - W(k - 2)) - 3.0 * (W(k) - W(k - 1)), 12.0, R12);
    return flux4 + sgn(-vel) * corr;
  }
  if (k == nz && !c.top_lid) return 0.5 * (W(nz) + W(nz - 1));
  return 0.0;
}
__device__ __forceinline__ double wflux(const Grid &g, const WColumn &c, int k, int j, int i) {
  const int nz = g.nz;
  if (k < 1 || k > nz || (k == nz && c.top_lid)) return 0.0;
  const double vel = wvel(g, c, k, j, i);
  auto W = [&](int kk) { return ld(c.w, ix3(kk, j, i, g.ny, g.nx)); };
  if (k == 1) return vel * 0.5 * (W(1) + W(0));
  if (k == nz) return vel * 0.5 * (W(nz) + W(nz - 1));
  return flux3v(W(k - 2), W(k - 1), W(k), W(k + 1), vel);
}

// g.nz here is the mass level count; w has g.nz + 1 levels
__global__ void k_vdiv_w(Grid g, WColumn c, double *tend) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  double t = 0.0;
  if (k >= 1 && k <= nz - 1) t = -ld(g.rdn, k) * (wflux(g, c, k + 1, j, i) - wflux(g, c, k, j, i));
  if (k == nz && !c.top_lid) t = t + 2.0 * ld(g.rdn, nz - 1) * wflux(g, c, nz, j, i);
  tend[ix3(k, j, i, ny, nx)] = t;
}

// Its VJP: Fbar(k) = rdn(k) lam(k) [k <= nz-1] - rdn(k-1) lam(k-1) [k >= 2]
// + 2 rdn(nz-1) lam(nz) [k = nz, open top]; w_bar(l) gathers
// Fbar(k) vel(k) dh_k/dw(l) over the faces k = l-1 .. l+2 whose stencils hold
// level l; velbar(k) = Fbar(k) h_k(w) and rom_bar(l) = (velbar(l) +
// velbar(l+1)) / 2.  Outputs given as NULL are skipped.
__global__ void k_vdiv_w_vjp(Grid g, WColumn c, const double *lam, double *w_bar, double *rom_bar) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int l = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  auto L = [&](int kk) { return ld(lam, ix3(kk, j, i, ny, nx)); };
  auto fbar = [&](int k) {
    double f = 0.0;
    if (k <= nz - 1) f += ld(g.rdn, k) * L(k);
    if (k >= 2) f -= ld(g.rdn, k - 1) * L(k - 1);
    if (k == nz && !c.top_lid) f += 2.0 * ld(g.rdn, nz - 1) * L(nz);
    return f;
  };
  auto live = [&](int k) { return k >= 1 && k <= nz && !(k == nz && c.top_lid); };
  if (w_bar != nullptr) {
    double acc = 0.0;
    for (int k = l - 1; k <= l + 2; ++k) {
      if (!live(k)) continue;
      const double vel = wvel(g, c, k, j, i);
      double wt = 0.0;
      if (k == 1 || k == nz) {
        wt = (l == k || l == k - 1) ? 0.5 : 0.0;
      } else {
        const double s = sgn(-vel);
        switch (l - (k - 2)) {  // stencil w(k-2) .. w(k+1)
          case 0: wt = w3<0>(s); break;
          case 1: wt = w3<1>(s); break;
          case 2: wt = w3<2>(s); break;
          default: wt = w3<3>(s); break;
        }
      }
      acc += fbar(k) * vel * wt;
    }
    w_bar[ix3(l, j, i, ny, nx)] = acc;
  }
  if (rom_bar != nullptr) {
    auto velbar = [&](int k) { return live(k) ? fbar(k) * wface(g, c, k, j, i, wvel(g, c, k, j, i)) : 0.0; };
    rom_bar[ix3(l, j, i, ny, nx)] = 0.5 * (velbar(l) + velbar(l + 1));
  }
}

}  // namespace wg
