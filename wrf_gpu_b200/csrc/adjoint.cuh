// Flux-form scalar advection operator (h5/v3, periodic) and its hand-written
// adjoint with respect to the advected field.
//
// For fixed transport velocities (ru, rv at the cells' west / south faces,
// rom at the w faces) the tendency tend = L(ru, rv, rom) q of
// flux_advection.py:482-568 is linear in q: the upwind switch sign(vel)
// depends on the velocity only.  k_scalar_adv_op applies L; k_scalar_adv_adj
// applies its transpose L^T to a tendency-space vector lambda:
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

namespace wg {

struct AdvOpArgs {
  const double *ru, *rv, *rom;  // (nz, ny, nx), (nz, ny, nx), (nz+1, ny, nx)
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
  const double msftx = ld(g.msftx, ix2(j, i, nx));
  double t = -msftx * g.rdx * (fx(i + 1) - fx(i));
  t = t - msftx * g.rdy * (fy(j + 1) - fy(j));
  auto qc = [&](int kk) { return ld(q, ix3(kk, j, i, ny, nx)); };
  const double v1 = (k + 1 <= nz - 1) ? vflux3_at(g, k + 1, ld(v.rom, ix3(k + 1, j, i, ny, nx)), qc) : 0.0;
  const double v0 = (k >= 1) ? vflux3_at(g, k, ld(v.rom, ix3(k, j, i, ny, nx)), qc) : 0.0;
  tend[ix3(k, j, i, ny, nx)] = t - ld(g.rdnw, k) * (v1 - v0);
}

// flux5 weight of stencil position m (0..5 = q-3..q+2) for upwind sign s.
__device__ __forceinline__ double w5(int m, double s) {
  switch (m) {
    case 0: return (1.0 + s) / 60.0;
    case 1: return (-8.0 - 5.0 * s) / 60.0;
    case 2: return (37.0 + 10.0 * s) / 60.0;
    case 3: return (37.0 - 10.0 * s) / 60.0;
    case 4: return (-8.0 + 5.0 * s) / 60.0;
    default: return (1.0 - s) / 60.0;
  }
}
// flux3 weight of stencil position m (0..3 = q(m-2)..q(m+1)) for s' = sign(-vel).
__device__ __forceinline__ double w3(int m, double s) {
  switch (m) {
    case 0: return (-1.0 - s) / 12.0;
    case 1: return (7.0 + 3.0 * s) / 12.0;
    case 2: return (7.0 - 3.0 * s) / 12.0;
    default: return (-1.0 + s) / 12.0;
  }
}

__global__ void k_scalar_adv_adj(Grid g, AdvOpArgs v, const double *lam, double *qbar) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  double acc = 0.0;
  // x faces ii = i-2 .. i+3 (west faces of cells ii); this cell is stencil
  // position 3 - t of face ii = i + t.  ml[t+3] = msftx * lambda at cell i+t.
  {
    double ml[7];
#pragma unroll
    for (int t = -3; t <= 3; ++t) {
      const int ii = wrp(i + t, nx);
      ml[t + 3] = ld(g.msftx, ix2(j, ii, nx)) * ld(lam, ix3(k, j, ii, ny, nx));
    }
#pragma unroll
    for (int t = -2; t <= 3; ++t) {
      const double vel = ld(v.ru, ix3(k, j, wrp(i + t, nx), ny, nx));
      acc += vel * w5(3 - t, sgn(vel)) * (g.rdx * (ml[t + 3] - ml[t + 2]));
    }
  }
  {
    double ml[7];
#pragma unroll
    for (int t = -3; t <= 3; ++t) {
      const int jj = wrp(j + t, ny);
      ml[t + 3] = ld(g.msftx, ix2(jj, i, nx)) * ld(lam, ix3(k, jj, i, ny, nx));
    }
#pragma unroll
    for (int t = -2; t <= 3; ++t) {
      const double vel = ld(v.rv, ix3(k, wrp(j + t, ny), i, ny, nx));
      acc += vel * w5(3 - t, sgn(vel)) * (g.rdy * (ml[t + 3] - ml[t + 2]));
    }
  }
  // z faces m = 1 .. nz-1 whose stencil holds level k
  auto Lz = [&](int kk) { return ld(lam, ix3(kk, j, i, ny, nx)); };
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
  qbar[ix3(k, j, i, ny, nx)] = acc;
}

// The full vector-Jacobian product.  tend is bilinear in (q, vel): with the
// upwind signs frozen each face flux is F_f = vel_f h_f(q), so besides
// q_bar (as k_scalar_adv_adj)
//   velbar_f = Fbar_f h_f(q),   h_f = flux5 / flux3 of the face's stencil
//   (the second-order face value at m = 1 and nz-1),
//   Fbar_x(i) = rdx (msftx(i) lam(i) - msftx(i-1) lam(i-1)), likewise y,
//   Fbar_z(m) = rdnw(m) lam(m) - rdnw(m-1) lam(m-1).
// Index space (nx, ny, nz+1): q_bar, ru_bar, rv_bar at cell (k, j, i) and
// the west / south face of it for k < nz, rom_bar at w face (k, j, i) (zero
// at k = 0 and nz, whose fluxes are zero).  Outputs given as NULL are
// skipped; the shared loads (lam, msftx, the velocities) are made once.
__global__ void k_scalar_adv_vjp(Grid g, AdvOpArgs v, const double *q, const double *lam, double *q_bar,
                                 double *ru_bar, double *rv_bar, double *rom_bar) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  auto Q = [&](int jj, int ii) { return ld(q, ix3(k, wrp(jj, ny), wrp(ii, nx), ny, nx)); };
  if (k < nz) {
    double acc = 0.0;
    {
      double ml[7];
#pragma unroll
      for (int t = -3; t <= 3; ++t) {
        const int ii = wrp(i + t, nx);
        ml[t + 3] = ld(g.msftx, ix2(j, ii, nx)) * ld(lam, ix3(k, j, ii, ny, nx));
      }
      double vel0 = 0.0;
#pragma unroll
      for (int t = -2; t <= 3; ++t) {
        const double vel = ld(v.ru, ix3(k, j, wrp(i + t, nx), ny, nx));
        if (t == 0) vel0 = vel;
        acc += vel * w5(3 - t, sgn(vel)) * (g.rdx * (ml[t + 3] - ml[t + 2]));
      }
      if (ru_bar != nullptr)
        ru_bar[ix3(k, j, i, ny, nx)] =
            g.rdx * (ml[3] - ml[2]) * flux5(Q(j, i - 3), Q(j, i - 2), Q(j, i - 1), Q(j, i), Q(j, i + 1), Q(j, i + 2), vel0);
    }
    {
      double ml[7];
#pragma unroll
      for (int t = -3; t <= 3; ++t) {
        const int jj = wrp(j + t, ny);
        ml[t + 3] = ld(g.msftx, ix2(jj, i, nx)) * ld(lam, ix3(k, jj, i, ny, nx));
      }
      double vel0 = 0.0;
#pragma unroll
      for (int t = -2; t <= 3; ++t) {
        const double vel = ld(v.rv, ix3(k, wrp(j + t, ny), i, ny, nx));
        if (t == 0) vel0 = vel;
        acc += vel * w5(3 - t, sgn(vel)) * (g.rdy * (ml[t + 3] - ml[t + 2]));
      }
      if (rv_bar != nullptr)
        rv_bar[ix3(k, j, i, ny, nx)] =
            g.rdy * (ml[3] - ml[2]) * flux5(Q(j - 3, i), Q(j - 2, i), Q(j - 1, i), Q(j, i), Q(j + 1, i), Q(j + 2, i), vel0);
    }
    if (q_bar != nullptr) {
      auto Lz = [&](int kk) { return ld(lam, ix3(kk, j, i, ny, nx)); };
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
          wk = w3(2 - t, sgn(-rom));
        }
        acc += rom * wk * (ld(g.rdnw, m) * Lz(m) - ld(g.rdnw, m - 1) * Lz(m - 1));
      }
      q_bar[ix3(k, j, i, ny, nx)] = acc;
    }
  }
  if (rom_bar != nullptr) {
    double r = 0.0;
    if (k >= 1 && k <= nz - 1) {
      auto qc = [&](int kk) { return ld(q, ix3(kk, j, i, ny, nx)); };
      auto L = [&](int kk) { return ld(lam, ix3(kk, j, i, ny, nx)); };
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

}  // namespace wg
