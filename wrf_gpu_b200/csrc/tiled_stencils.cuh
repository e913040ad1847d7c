// Shared-memory plane tiles for the horizontal-stencil stage kernels, and the
// per-level pieces of the PD / monotonic limiter that the marching kernels
// (tiled_march.cuh) assemble.
//
// A tile covers 32 x 8 cells of one level plus a halo: element (r, c) of a
// (8 + 2*HY) x (32 + 2*HX) tile holds the field at the periodically wrapped
// cell (j0 - HY + r, i0 - HX + c), so the flux stencils read shared memory at
// fixed offsets.  The arithmetic keeps the reference's expression order.
#pragma once
#include "dycore_common.cuh"
#include "stage_kernels.cuh"

namespace wg {

constexpr int TSX = 32;
constexpr int TSY = 8;

template <int HX, int HY>
struct Tile {
  static constexpr int W = TSX + 2 * HX;
  static constexpr int H = TSY + 2 * HY;
  static constexpr int N = W * H;
};

// Stage one plane tile: element (r, c) holds src[wrap(j0-HY+r), wrap(i0-HX+c)] - sub.
template <int HX, int HY>
__device__ __forceinline__ void load_tile(double *t, const double *plane, int pitch, int i0, int j0, int px, int py,
                                          double sub) {
  using T = Tile<HX, HY>;
  for (int e = threadIdx.y * TSX + threadIdx.x; e < T::N; e += TSX * TSY) {
    const int r = e / T::W, c = e - r * T::W;
    const int jj = wrp(j0 - HY + r, py), ii = wrp(i0 - HX + c, px);
    t[e] = __ldg(plane + (size_t)jj * pitch + ii) - sub;
  }
}

// ---------------------------------------------------------------------------
// PD / monotonic limited scalar advection (flux_advection.py:736-1000):
// per-level face fluxes, cell scales and limited tendency.
// ---------------------------------------------------------------------------
// Vertical spacing of the two faces of the block's level (k and k+1):
// dz = 2/(rdnw[m] + rdnw[m-1]) (flux_advection.py upwind z flux), its
// correctly rounded reciprocal and dz/dt.  Computed once per block.
struct ZConst {
  double dz, rdz, dz_dt;
};

struct LimTiles {
  double *q;    // Tile<3,3>: field - offset
  double *qo;   // Tile<1,1>: field_old - offset
  double *ru;   // Tile<1,0>
  double *rv;   // Tile<0,1>
  double *mt;   // Tile<1,1>: current total dry mass (2-D)
  const struct ZConst *zc;  // the level's two faces: dz, 1/dz, dz/dt
  // low-order and antidiffusive fluxes of the tile's x faces (TSY rows of
  // TSX+1 faces) and y faces (TSY+1 rows of TSX faces), each computed once
  double *fxl, *fxa, *fyl, *fya;
};

constexpr int LIM_NXF = TSY * (TSX + 1);
constexpr int LIM_NYF = (TSY + 1) * TSX;

__device__ __forceinline__ void lim_zconst(const Grid &g, const LimArgs &a, int k, ZConst *zc) {
  const int f = threadIdx.y * TSX + threadIdx.x;
  if (f < 2) {
    const int m = k + f;
    ZConst z{1.0, 1.0, 1.0};
    if (m >= 1 && m < g.nz) {
      z.dz = 2.0 / (ld(g.rdnw, m) + ld(g.rdnw, m - 1));
      z.rdz = 1.0 / z.dz;
      z.dz_dt = z.dz / a.dt;
    }
    zc[f] = z;
  }
}

// Low-order upwind (flux_advection.py:614-675) and antidiffusive (high
// order :678-711 minus low order) fluxes of every x and y face of the tile,
// one face per thread item, into shared memory.  Edge tiles compute a few
// harmless extra faces from the periodically wrapped staged values.  SUB
// false: the field's offset is +0.0 and the staged values are read as they
// are (x - 0.0 == x bit for bit).
template <typename F, bool DEG, bool SUB = true>
__device__ __forceinline__ void lim_face_fluxes(const Grid &g, const LimArgs &a, const LimTiles &t, int k, int i0,
                                                int j0) {
  using TQ = Tile<3, 3>;
  using TO = Tile<1, 1>;
  using TR = Tile<1, 0>;
  using TV = Tile<0, 1>;
  const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
  auto Q = [&](int r, int cc) {
    const double x = t.q[(r + 3) * TQ::W + (cc + 3)];
    return SUB ? x - a.offset : x;
  };
  auto QO = [&](int r, int cc) {
    const double x = t.qo[(r + 1) * TO::W + (cc + 1)];
    return SUB ? x - a.offset : x;
  };
  auto MT = [&](int r, int cc) { return t.mt[(r + 1) * TO::W + (cc + 1)]; };
  // cr = vel*dt/dxy/mu_face and mu_face*(dxy/dt)*(...) with the constant
  // divisions done by div_rcp / per-launch constants (same bits).
  auto upw = [&](double fo_m1, double fo_0, double vel, double mu_face, double dxy, double rdxy, double dxy_dt) {
    double cr = div_rcp(vel * a.dt, dxy, rdxy) / mu_face;
    double ab = fabs(cr);
    return mu_face * dxy_dt * (0.5 * dmin(1.0, cr + ab) * fo_m1 + 0.5 * dmax(-1.0, cr - ab) * fo_0);
  };
  for (int e = threadIdx.y * TSX + threadIdx.x; e < LIM_NXF + LIM_NYF; e += TSX * TSY) {
    if (e < LIM_NXF) {
      const int r = e / (TSX + 1), m = e - r * (TSX + 1);  // x face at local column m of row r
      const double vel = t.ru[r * TR::W + (m + 1)];
      const double muu = 0.5 * (MT(r, m) + MT(r, m - 1));
      const double mu_u = c1 * muu + c2;
      // the specified degradation: tiered high-order faces, no low-order
      // flux on face 0 (nor on face nx, its wrap)
      const int gm = i0 + m;
      const double lo = (DEG && (gm == 0 || gm == g.nx)) ? 0.0 : upw(QO(r, m - 1), QO(r, m), vel, mu_u, a.dxl, a.rdxl, a.dxl_dt);
      const double hi = DEG ? hflux_spec<F>(gm, g.nx, false, vel, Q(r, m - 3), Q(r, m - 2), Q(r, m - 1), Q(r, m),
                                              Q(r, m + 1), Q(r, m + 2))
                              : hflux5<F>(vel, Q(r, m - 3), Q(r, m - 2), Q(r, m - 1), Q(r, m), Q(r, m + 1), Q(r, m + 2));
      t.fxl[e] = lo;
      t.fxa[e] = hi - lo;
    } else {
      const int e2 = e - LIM_NXF;
      const int r = e2 / TSX, cc = e2 - r * TSX;  // y face at local row r of column cc
      const double vel = t.rv[(r + 1) * TV::W + cc];
      const double muv = 0.5 * (MT(r, cc) + MT(r - 1, cc));
      const double mu_v = c1 * muv + c2;
      const int gm = j0 + r;
      const double lo = (DEG && (gm == 0 || gm == g.ny)) ? 0.0 : upw(QO(r - 1, cc), QO(r, cc), vel, mu_v, a.dyl, a.rdyl, a.dyl_dt);
      const double hi = DEG ? hflux_spec<F>(gm, g.ny, false, vel, Q(r - 3, cc), Q(r - 2, cc), Q(r - 1, cc), Q(r, cc),
                                              Q(r + 1, cc), Q(r + 2, cc))
                              : hflux5<F>(vel, Q(r - 3, cc), Q(r - 2, cc), Q(r - 1, cc), Q(r, cc), Q(r + 1, cc), Q(r + 2, cc));
      t.fyl[e2] = lo;
      t.fya[e2] = hi - lo;
    }
  }
}

// The 12 face fluxes of cell (k, j, i) from the staged tiles: low-order
// upwind (flux_advection.py:614-675) and antidiffusive = high order
// (:678-711) minus low order, at the cell's two x, y and z faces.
// With have_z0 the bottom-face z fluxes are taken from cf.lz0/cf.az0 (carried
// up from the level below) instead of being recomputed.
template <typename F>
__device__ __forceinline__ void cell_fluxes_tiled(const Grid &g, const LimArgs &a, const LimTiles &t, int k, int j,
                                                  int i, const double *field, const double *field_old,
                                                  CellFluxes &cf, bool have_z0 = false) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tx = threadIdx.x, ty = threadIdx.y;
  using TO = Tile<1, 1>;
  auto MT = [&](int r, int cc) { return t.mt[(r + 1) * TO::W + (cc + 1)]; };
  auto qf = [&](int kk) { return ld(field, ix3(kk, j, i, ny, nx)) - a.offset; };
  auto qo = [&](int kk) { return ld(field_old, ix3(kk, j, i, ny, nx)) - a.offset; };
  auto zf = [&](int m, double &lo, double &an) {
    if (m <= 0 || m >= nz) {
      lo = 0.0;
      an = 0.0;
      return;
    }
    const double romv = ld(a.rom, ix3(m, j, i, ny, nx));
    const double mtc = MT(ty, tx);
    const double muh_m = ld(g.c1h, m) * mtc + ld(g.c2h, m);
    const double muh_mm1 = ld(g.c1h, m - 1) * mtc + ld(g.c2h, m - 1);
    const int zi = m - k;  // 0: bottom face of this level, 1: top face
    const double mu_face = 0.5 * (muh_m + muh_mm1);
    const double cr = div_rcp(romv * a.dt, t.zc[zi].dz, t.zc[zi].rdz) / mu_face;
    const double ab = fabs(cr);
    lo = mu_face * t.zc[zi].dz_dt * (0.5 * dmin(1.0, cr + ab) * qo(m - 1) + 0.5 * dmax(-1.0, cr - ab) * qo(m));
    const double hi = vflux3_at<F>(g, m, romv, qf);
    an = hi - lo;
  };
  const int x0 = ty * (TSX + 1) + tx, y0 = ty * TSX + tx;
  cf.lx0 = t.fxl[x0]; cf.ax0 = t.fxa[x0];
  cf.lx1 = t.fxl[x0 + 1]; cf.ax1 = t.fxa[x0 + 1];
  cf.ly0 = t.fyl[y0]; cf.ay0 = t.fya[y0];
  cf.ly1 = t.fyl[y0 + TSX]; cf.ay1 = t.fya[y0 + TSX];
  if (!have_z0) zf(k, cf.lz0, cf.az0);
  zf(k + 1, cf.lz1, cf.az1);
}

// Scale(s) of the PD (opt 1) / monotonic (opt 2) limiter at cell (k, j, i)
// from its 12 face fluxes (flux_advection.py:736-935).
__device__ __forceinline__ void lim_cell_scales(const Grid &g, const LimArgs &a, const LimTiles &t, int k, int j,
                                                int i, const double *field_old, const CellFluxes &cf, double &r1,
                                                double &r2) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tx = threadIdx.x, ty = threadIdx.y;
  using TO = Tile<1, 1>;
  auto QO = [&](int r, int cc) { return t.qo[(r + 1) * TO::W + (cc + 1)] - a.offset; };
  const double msftx = ld(g.msftx, ix2(j, i, nx));
  const double rdzw = ld(g.rdnw, k);
  const double mass_old = ld(g.c1h, k) * ld(a.mu_old, ix2(j, i, nx)) + ld(g.c2h, k);
  const double fo = QO(ty, tx);
  const double div_low = msftx * msftx * (g.rdx * (cf.lx1 - cf.lx0) + g.rdy * (cf.ly1 - cf.ly0)) +
                         msftx * rdzw * (cf.lz1 - cf.lz0);
  const double ph_low = mass_old * fo - a.dt * div_low;
  auto pos = [](double x) { return dmax(0.0, x); };
  auto neg = [](double x) { return dmin(0.0, x); };
  const double flux_out = a.dt * (msftx * msftx * (g.rdx * (pos(cf.ax1) - neg(cf.ax0)) + g.rdy * (pos(cf.ay1) - neg(cf.ay0))) +
                                  msftx * rdzw * (neg(cf.az1) - pos(cf.az0)));
  if (a.opt == 1) {
    r1 = (flux_out > ph_low) ? dmax(0.0, ph_low / (flux_out + PD_EPS)) : 1.0;
    r2 = r1;
  } else {
    auto qov = [&](int kk) { return ld(field_old, ix3(kk, j, i, ny, nx)) - a.offset; };
    double qmax = fo, qmin = fo;
    const double n0 = QO(ty, tx - 1), n1 = QO(ty, tx + 1), n2 = QO(ty - 1, tx), n3 = QO(ty + 1, tx);
    const double n4 = (k == 0) ? fo : qov(k - 1), n5 = (k == nz - 1) ? fo : qov(k + 1);
    qmax = dmax(qmax, dmax(n0, n1));
    qmin = dmin(qmin, dmin(n0, n1));
    qmax = dmax(qmax, dmax(n2, n3));
    qmin = dmin(qmin, dmin(n2, n3));
    qmax = dmax(qmax, dmax(n4, n5));
    qmin = dmin(qmin, dmin(n4, n5));
    const double flux_in = -a.dt * (msftx * msftx * (g.rdx * (neg(cf.ax1) - pos(cf.ax0)) + g.rdy * (neg(cf.ay1) - pos(cf.ay0))) +
                                    msftx * rdzw * (pos(cf.az1) - neg(cf.az0)));
    const double ph_hi = qmax * mass_old - ph_low;
    const double ph_lo = ph_low - qmin * mass_old;
    r1 = (flux_in > ph_hi) ? dmax(0.0, ph_hi / (flux_in + PD_EPS)) : 1.0;
    r2 = (flux_out > ph_lo) ? dmax(0.0, ph_lo / (flux_out + PD_EPS)) : 1.0;
  }
}

// West / south / bottom face fluxes of every cell (low order l*, antidiffusive
// a*), written by the limiter's scale pass so the tendency pass reads them
// instead of recomputing them; the east / north / top faces of a cell are the
// west / south / bottom faces of its neighbours (the top face of level nz-1
// carries no flux).
// Stored as T: float64, or float32 in the mixed-precision variant (whose
// advective fluxes are FP32 quantities).
template <typename T>
struct LimFacesT {
  T *lx, *ax, *ly, *ay, *lz, *az;
};
using LimFaces = LimFacesT<double>;

// Limited tendency at cell (k, j, i) (flux_advection.py:937-1000) from its
// face fluxes; S1(dr, dc) / S2(dr, dc) return the scales at the horizontal
// neighbour (j + dr, i + dc) of level k, s1 / s2 are the scale arrays (for the
// levels above and below).
template <typename SA1, typename SA2, typename T>
__device__ __forceinline__ double lim_cell_tend(const Grid &g, const LimArgs &a, SA1 S1, SA2 S2, int k, int j, int i,
                                                const T *s1, const T *s2, const CellFluxes &cf) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  auto S1k = [&](int kk) { return ld(s1, ix3(kk, j, i, ny, nx)); };
  auto S2k = [&](int kk) { return ld(s2, ix3(kk, j, i, ny, nx)); };
  double fx0, fx1, fy0, fy1, fz0, fz1;
  if (a.opt == 1) {
    auto limh = [&](double A, double s_m1, double s_c) { return A > 0.0 ? s_m1 * A : (A < 0.0 ? s_c * A : A); };
    fx0 = limh(cf.ax0, S1(0, -1), S1(0, 0));
    fx1 = limh(cf.ax1, S1(0, 0), S1(0, 1));
    fy0 = limh(cf.ay0, S1(-1, 0), S1(0, 0));
    fy1 = limh(cf.ay1, S1(0, 0), S1(1, 0));
    auto limz = [&](double A, double below, double above) { return A < 0.0 ? below * A : (A > 0.0 ? above * A : A); };
    const double sc = S1(0, 0);
    fz0 = limz(cf.az0, k == 0 ? sc : S1k(k - 1), sc);
    fz1 = limz(cf.az1, sc, k + 1 >= nz ? sc : S1k(k + 1));
  } else {
    auto limh = [&](double A, double in_c, double out_c, double in_m1, double out_m1) {
      return A > 0.0 ? dmin(in_c, out_m1) * A : dmin(out_c, in_m1) * A;
    };
    fx0 = limh(cf.ax0, S1(0, 0), S2(0, 0), S1(0, -1), S2(0, -1));
    fx1 = limh(cf.ax1, S1(0, 1), S2(0, 1), S1(0, 0), S2(0, 0));
    fy0 = limh(cf.ay0, S1(0, 0), S2(0, 0), S1(-1, 0), S2(-1, 0));
    fy1 = limh(cf.ay1, S1(1, 0), S2(1, 0), S1(0, 0), S2(0, 0));
    auto limz = [&](double A, double in_above, double out_above, double in_below, double out_below) {
      return A < 0.0 ? dmin(in_above, out_below) * A : dmin(out_above, in_below) * A;
    };
    const int kb = (k == 0) ? 0 : k - 1;
    const int ka = (k + 1 >= nz) ? nz - 1 : k + 1;
    const double s1c = S1(0, 0), s2c = S2(0, 0);
    const double s1b = (kb == k) ? s1c : S1k(kb), s2b = (kb == k) ? s2c : S2k(kb);
    const double s1a = (ka == k) ? s1c : S1k(ka), s2a = (ka == k) ? s2c : S2k(ka);
    fz0 = limz(cf.az0, s1c, s2c, s1b, s2b);
    fz1 = limz(cf.az1, s1a, s2a, s1c, s2c);
  }
  fx0 = fx0 + cf.lx0;
  fx1 = fx1 + cf.lx1;
  fy0 = fy0 + cf.ly0;
  fy1 = fy1 + cf.ly1;
  fz0 = fz0 + cf.lz0;
  fz1 = fz1 + cf.lz1;
  const double msftx = ld(g.msftx, ix2(j, i, nx));
  const bool xin = !a.deg || (i >= 1 && i <= nx - 2), yin = !a.deg || (j >= 1 && j <= ny - 2);
  double tend = -msftx * g.rdx * (xin ? (fx1 - fx0) : 0.0);
  tend = tend - msftx * g.rdy * (yin ? (fy1 - fy0) : 0.0);
  tend = tend - ld(g.rdnw, k) * (fz1 - fz0);
  return tend;
}

// The limiter's tendency pass, one thread per cell, from the face fluxes and
// scales the scale pass stored.
// T: the storage type of the face fluxes and scales; TO: of the tendency
// (float64 for theta, T for the moisture species).
template <typename T, typename TO>
__global__ void k_lim_tend_faces(Grid g, LimArgs a, LimFacesT<T> fc, const T *s1, const T *s2,
                                 const double *base, const double *mu_total_stage, TO *tend_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i >= nx || j >= ny) return;
  const size_t c = ix3(k, j, i, ny, nx);
  const size_t ce = ix3(k, j, wrp(i + 1, nx), ny, nx), cn = ix3(k, wrp(j + 1, ny), i, ny, nx);
  CellFluxes cf;
  cf.lx0 = ld(fc.lx, c); cf.ax0 = ld(fc.ax, c); cf.lx1 = ld(fc.lx, ce); cf.ax1 = ld(fc.ax, ce);
  cf.ly0 = ld(fc.ly, c); cf.ay0 = ld(fc.ay, c); cf.ly1 = ld(fc.ly, cn); cf.ay1 = ld(fc.ay, cn);
  cf.lz0 = ld(fc.lz, c); cf.az0 = ld(fc.az, c);
  if (k + 1 < nz) {
    const size_t cu = ix3(k + 1, j, i, ny, nx);
    cf.lz1 = ld(fc.lz, cu);
    cf.az1 = ld(fc.az, cu);
  } else {
    cf.lz1 = 0.0;
    cf.az1 = 0.0;
  }
  auto S1 = [&](int dr, int dc) { return ld(s1, ix3(k, wrp(j + dr, ny), wrp(i + dc, nx), ny, nx)); };
  auto S2 = [&](int dr, int dc) { return ld(s2, ix3(k, wrp(j + dr, ny), wrp(i + dc, nx), ny, nx)); };
  const double tend = lim_cell_tend(g, a, S1, S2, k, j, i, s1, s2, cf);
  if (base != nullptr) {
    const double mass_h = ld(g.c1h, k) * ld(mu_total_stage, ix2(j, i, nx)) + ld(g.c2h, k);
    tend_out[c] = (TO)(ld(base, c) * mass_h + tend);
  } else {
    tend_out[c] = (TO)tend;
  }
}

}  // namespace wg
