// Level-marching tiled stencil kernels with asynchronous tile staging.
//
// A block owns one 32 x 8 tile of the horizontal grid and marches up a chunk
// of levels.  The plane tiles a level needs are copied into shared memory
// with cp.async (8-byte asynchronous global->shared copies, which need no
// registers and work for any row alignment -- the grid's odd row pitch rules
// out tensor-map TMA), double-buffered so level k+1's copies are in flight
// while level k is computed.  The periodic wrap of every staged element is
// resolved once per block into per-thread plane offsets.  Vertical fluxes are
// carried up the march: face k+1 of level k is face k of level k+1.
// Arithmetic keeps the reference's expression order.
#pragma once
#include <type_traits>
#include "dycore_common.cuh"
#include "stage_kernels.cuh"
#include "tiled_stencils.cuh"

namespace wg {

// Per-thread share of one (TSY + 2*HY) x (TSX + 2*HX) plane tile: the
// elements e = tid, tid + 256, ... with their wrapped in-plane offsets.
template <int HX, int HY>
struct TileSlots {
  static constexpr int NS = (Tile<HX, HY>::N + TSX * TSY - 1) / (TSX * TSY);
  int off[NS];
  __device__ __forceinline__ void init(int i0, int j0, int pitch, int px, int py) {
    using T = Tile<HX, HY>;
    const int tid = threadIdx.y * TSX + threadIdx.x;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      const int e = tid + n * TSX * TSY;
      off[n] = -1;
      if (e < T::N) {
        const int r = e / T::W, c = e - r * T::W;
        off[n] = wrp(j0 - HY + r, py) * pitch + wrp(i0 - HX + c, px);
      }
    }
  }
  // Issue the copies of this thread's elements of the tile of `plane`.
  __device__ __forceinline__ void issue(double *tile, const double *plane) const {
    const int tid = threadIdx.y * TSX + threadIdx.x;
#pragma unroll
    for (int n = 0; n < NS; ++n)
      if (off[n] >= 0) cp_async8(tile + tid + n * TSX * TSY, plane + off[n]);
  }
};

// p[n] for a runtime n, by compares (keeps a by-value pointer array out of
// local memory).
template <typename P>
__device__ __forceinline__ P pick6(const P (&p)[6], int n) {
  P r = p[0];
#pragma unroll
  for (int t = 1; t < 6; ++t)
    if (n == t) r = p[t];
  return r;
}

// Resident 256-thread blocks per SM requested from the register allocator
// (timed at 433 x 433 x 50: 5 for the scalar advection -- 2.19 vs 2.26
// ms/step at 6, 2.43 at 7 --, 4 for the limiter's six-species scale pass --
// 2.10 vs 2.22 ms/step at 5, 2.48 at 6, 2.44 at 3; unset: no request).
#ifndef WG_SCALAR_MINB
#define WG_SCALAR_MINB 5
#endif
#ifndef WG_LIM_MINB
#define WG_LIM_MINB 4
#endif
#ifdef WG_SCALAR_MINB
#define WG_SCALAR_BOUNDS __launch_bounds__(TSX * TSY, WG_SCALAR_MINB)
#else
#define WG_SCALAR_BOUNDS __launch_bounds__(TSX * TSY)
#endif
#ifdef WG_LIM_MINB
#define WG_LIM_BOUNDS __launch_bounds__(TSX * TSY, WG_LIM_MINB)
#else
#define WG_LIM_BOUNDS __launch_bounds__(TSX * TSY)
#endif

// Levels per marching block: the kernels are instantiated for these chunk
// sizes (compile-time loop bounds); the default and the tuner's choices.
constexpr int MARCH_KC = 10;
constexpr int MARCH_KC_CHOICES[] = {5, 10, 25};

// ---------------------------------------------------------------------------
// Plain h5/v3 scalar advection (flux_advection.py:482-568) of theta and the
// moisture species, and theta_work (small_step_prep.py:321).  blockIdx.z =
// chunk * nfields + field, so the fields of one chunk run together and share
// the transport-velocity tiles in L2; field 0 is theta (theta_work is always
// written, the tendency only when theta is not limited), fields 1..6 the
// species.
// ---------------------------------------------------------------------------
template <typename F, int KC, bool DEG>
__global__ void WG_SCALAR_BOUNDS k_scalar_adv_march(Grid g, StateR s, StateR ref, const double *ru,
                                                                const double *rv, const double *rom, const double *mut,
                                                                const double *muts0, const double *base_theta,
                                                                int theta_plain, int nfields, MassOut o) {
  using TQ = Tile<3, 3>;
  using TR = Tile<1, 0>;
  using TV = Tile<0, 1>;
  constexpr int NXF = TSY * (TSX + 1);
  constexpr int NYF = (TSY + 1) * TSX;
  __shared__ double sq[2][TQ::N];
  __shared__ double sru[2][TR::N];
  __shared__ double srv[2][TV::N];
  __shared__ double sfx[NXF];
  __shared__ double sfy[NYF];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * TSX, j0 = blockIdx.y * TSY;
  const int chunk = blockIdx.z / nfields, field = blockIdx.z - chunk * nfields;
  const int k0 = chunk * KC, k1 = min(nz, k0 + KC);
  const int i = i0 + tx, j = j0 + ty;
  const bool valid = i < nx && j < ny;
  const double *fld = (field == 0) ? s.theta : pick6(s.q, field - 1);
  // the species' tendencies are stored as F (float32 in the mixed variant)
  F *q_out = (field == 0) ? nullptr : pick6(MassOutQ<F>::get(o), field - 1);
  const double sub = (field == 0) ? T0 : 0.0;
  const bool advect = (field > 0) || theta_plain;
  const size_t plane = (size_t)ny * nx;
  const size_t c2d = valid ? ix2(j, i, nx) : 0;
  const double msftx = valid ? ld(g.msftx, c2d) : 1.0;

  TileSlots<3, 3> slq;
  TileSlots<1, 0> slu;
  TileSlots<0, 1> slv;
  slq.init(i0, j0, nx, nx, ny);
  slu.init(i0, j0, nx, nx, ny);
  slv.init(i0, j0, nx, nx, ny);
  auto issue = [&](int k, int b) {
    slq.issue(sq[b], fld + (size_t)k * plane);
    slu.issue(sru[b], ru + (size_t)k * plane);
    slv.issue(srv[b], rv + (size_t)k * plane);
    cp_async_commit();
  };
  auto qc = [&](int kk) { return ld(fld, (size_t)kk * plane + c2d) - sub; };
  auto vflux = [&](int m) { return vflux3_at<F>(g, m, ld(rom, (size_t)m * plane + c2d), qc); };

  if (advect) issue(k0, 0);
  double v_lo = 0.0;  // vertical flux at the current level's bottom face
  if (advect && valid && k0 >= 1) v_lo = vflux(k0);
  for (int k = k0; k < k1; ++k) {
    const int b = (k - k0) & 1;
    if (advect) {
      if (k + 1 < k1) {
        issue(k + 1, b ^ 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
    }
    __syncthreads();
    double adv = 0.0;
    if (advect) {
      const double *Qt = sq[b];
      const double *RU = sru[b];
      const double *RV = srv[b];
      // SUB: theta's tiles less T0; the species' offset is 0 and x - 0.0 == x
      auto faces = [&](auto SUB) {
        auto Q = [&](int r, int cc) {
          const double x = Qt[(r + 3) * TQ::W + (cc + 3)];
          return decltype(SUB)::value ? x - sub : x;
        };
        for (int e = ty * TSX + tx; e < NXF + NYF; e += TSX * TSY) {
          if (e < NXF) {
            const int r = e / (TSX + 1), m = e - r * (TSX + 1);
            const double vel = RU[r * TR::W + (m + 1)];
            sfx[e] = DEG ? hflux_spec<F>(i0 + m, nx, false, vel, Q(r, m - 3), Q(r, m - 2), Q(r, m - 1), Q(r, m),
                                         Q(r, m + 1), Q(r, m + 2))
                         : hflux5<F>(vel, Q(r, m - 3), Q(r, m - 2), Q(r, m - 1), Q(r, m), Q(r, m + 1), Q(r, m + 2));
          } else {
            const int e2 = e - NXF;
            const int r = e2 / TSX, cc = e2 - r * TSX;
            const double vel = RV[(r + 1) * TV::W + cc];
            sfy[e2] = DEG ? hflux_spec<F>(j0 + r, ny, false, vel, Q(r - 3, cc), Q(r - 2, cc), Q(r - 1, cc),
                                          Q(r, cc), Q(r + 1, cc), Q(r + 2, cc))
                          : hflux5<F>(vel, Q(r - 3, cc), Q(r - 2, cc), Q(r - 1, cc), Q(r, cc), Q(r + 1, cc),
                                      Q(r + 2, cc));
          }
        }
      };
      if (field == 0)
        faces(std::true_type{});
      else
        faces(std::false_type{});
      __syncthreads();
      if (valid) {
        // the specified degradation leaves the outermost cells without
        // horizontal flux divergence (flux_advection.py:350-361)
        const bool xin = !DEG || (i >= 1 && i <= nx - 2), yin = !DEG || (j >= 1 && j <= ny - 2);
        double tend = -msftx * g.rdx * (xin ? (sfx[ty * (TSX + 1) + tx + 1] - sfx[ty * (TSX + 1) + tx]) : 0.0);
        tend = tend - msftx * g.rdy * (yin ? (sfy[(ty + 1) * TSX + tx] - sfy[ty * TSX + tx]) : 0.0);
        const double v_hi = (k + 1 <= nz - 1) ? vflux(k + 1) : 0.0;
        const double v0 = (k >= 1) ? v_lo : 0.0;
        adv = tend - ld(g.rdnw, k) * (v_hi - v0);
        v_lo = v_hi;
      }
    }
    if (valid) {
      const size_t c = (size_t)k * plane + c2d;
      if (field == 0) {
        if (theta_plain) {
          if (base_theta != nullptr) {
            const double mass_h = ld(g.c1h, k) * ld(s.mu_total, c2d) + ld(g.c2h, k);
            o.t_tend[c] = ld(base_theta, c) * mass_h + adv;
          } else {
            o.t_tend[c] = adv;
          }
        }
        const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
        const double mass_ref = c1 * ld(muts0, c2d) + c2;
        const double mass_cur = c1 * ld(mut, c2d) + c2;
        o.theta_w[c] = mass_ref * (ld(ref.theta, c) - T0) - mass_cur * (ld(s.theta, c) - T0);
      } else {
        q_out[c] = (F)adv;
      }
    }
    __syncthreads();  // sq/sru/srv[b] and sfx/sfy are reused next level
  }
}

inline int march_nchunk(int nz, int kc) { return (nz + kc - 1) / kc; }

// ---------------------------------------------------------------------------
// PD / monotonic limited scalar advection (flux_advection.py:736-1000): the
// marching scale pass.  Writes the per-cell scale(s) and the west / south /
// bottom face fluxes of every cell for the tendency pass (k_lim_tend_faces).
// The bottom-face z fluxes of a level are the top-face fluxes carried from
// the level below.
// ---------------------------------------------------------------------------
struct LimMarchSmem {
  double q[2][Tile<3, 3>::N];
  double qo[2][Tile<1, 1>::N];
  double ru[2][Tile<1, 0>::N];
  double rv[2][Tile<0, 1>::N];
  double mt[Tile<1, 1>::N];
  double fxl[LIM_NXF], fxa[LIM_NXF], fyl[LIM_NYF], fya[LIM_NYF];
  ZConst zc[2];
};

// Up to six fields limited in one launch (the moisture species of the final
// stage): field n's current and step-start values and its scratch (scales,
// face fluxes).  The field index is the fastest of blockIdx.x, so the fields'
// blocks of one tile run side by side and read the tile's transport
// velocities through L2 once.
template <typename F>
struct LimBatch {
  const double *field[6], *field_old[6];
  F *s1[6], *s2[6];
  LimFacesT<F> fo[6];
  int n;
};

template <typename F, int KC, bool DEG>
__global__ void WG_LIM_BOUNDS k_lim_march(Grid g, LimArgs a, LimBatch<F> lb) {
  __shared__ LimMarchSmem sm;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int bx = blockIdx.x / lb.n, fi = blockIdx.x - bx * lb.n;
  const double *field = pick6(lb.field, fi), *field_old = pick6(lb.field_old, fi);
  F *s1w = pick6(lb.s1, fi), *s2w = pick6(lb.s2, fi);
  LimFacesT<F> fo = lb.fo[0];
#pragma unroll
  for (int t = 1; t < 6; ++t)
    if (fi == t) fo = lb.fo[t];
  const int i0 = bx * TSX, j0 = blockIdx.y * TSY;
  const int k0 = blockIdx.z * KC, k1 = min(nz, k0 + KC);
  const int i = i0 + tx, j = j0 + ty;
  const bool valid = i < nx && j < ny;
  const size_t plane = (size_t)ny * nx;
  TileSlots<3, 3> slq;
  TileSlots<1, 1> slo;
  TileSlots<1, 0> slu;
  TileSlots<0, 1> slv;
  slq.init(i0, j0, nx, nx, ny);
  slo.init(i0, j0, nx, nx, ny);
  slu.init(i0, j0, nx, nx, ny);
  slv.init(i0, j0, nx, nx, ny);
  auto issue = [&](int k, int b) {
    const size_t o = (size_t)k * plane;
    slq.issue(sm.q[b], field + o);
    slo.issue(sm.qo[b], field_old + o);
    slu.issue(sm.ru[b], a.ru + o);
    slv.issue(sm.rv[b], a.rv + o);
    cp_async_commit();
  };
  load_tile<1, 1>(sm.mt, a.mut, nx, i0, j0, nx, ny, 0.0);  // 2-D, the same for every level
  issue(k0, 0);
  double zlo = 0.0, zan = 0.0;  // z fluxes of the current level's bottom face, carried up
  for (int k = k0; k < k1; ++k) {
    const int b = (k - k0) & 1;
    if (k + 1 < k1) {
      issue(k + 1, b ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    lim_zconst(g, a, k, sm.zc);
    __syncthreads();
    LimTiles t{sm.q[b], sm.qo[b], sm.ru[b], sm.rv[b], sm.mt, sm.zc, sm.fxl, sm.fxa, sm.fyl, sm.fya};
    if (__double_as_longlong(a.offset) == 0)
      lim_face_fluxes<F, DEG, false>(g, a, t, k, i0, j0);
    else
      lim_face_fluxes<F, DEG, true>(g, a, t, k, i0, j0);
    __syncthreads();
    if (valid) {
      CellFluxes cf;
      cf.lz0 = zlo;
      cf.az0 = zan;
      cell_fluxes_tiled<F>(g, a, t, k, j, i, field, field_old, cf, k > k0);
      zlo = cf.lz1;
      zan = cf.az1;
      const size_t c = (size_t)k * plane + ix2(j, i, nx);
      double r1, r2;
      lim_cell_scales(g, a, t, k, j, i, field_old, cf, r1, r2);
      s1w[c] = (F)r1;
      if (a.opt == 2) s2w[c] = (F)r2;  // the PD tendency reads s1 only
      fo.lx[c] = (F)cf.lx0;
      fo.ax[c] = (F)cf.ax0;
      fo.ly[c] = (F)cf.ly0;
      fo.ay[c] = (F)cf.ay0;
      fo.lz[c] = (F)cf.lz0;
      fo.az[c] = (F)cf.az0;
    }
    __syncthreads();  // staged tiles of buffer b, face fluxes and zc are reused next level
  }
}
}  // namespace wg
