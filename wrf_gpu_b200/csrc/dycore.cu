// Host orchestration and C ABI of the fp64 RK3 dycore step.
//
// One wrfgpu_rk3_step call replaces _rk_scan_step
// (src/gpuwrf/runtime/operational_mode.py:3319-3534): three RK stages of
// 1, ns/2 and ns acoustic substeps (operational_mode.py:3524-3530), each
// stage = stage kernels -> substep kernels -> finish kernels, all enqueued on
// the caller's stream with no host synchronisation or allocation.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>
#include <algorithm>

#include "../../include/wrfgpu.h"
#include "dycore_common.cuh"
#include "stage_kernels.cuh"
#include "acoustic_kernels.cuh"
#include "finish_kernels.cuh"
#include "column_tiled.cuh"
#include "column_stream.cuh"
#include "tiled_stencils.cuh"
#include "tiled_faces.cuh"
#include "tiled_march.cuh"
#include "adjoint.cuh"
#include "acoustic_adjoint.cuh"
#include "bdy_cadence.cuh"
#include "physics_merge.cuh"
#include "lbc.cuh"
#include "diffusion.cuh"
#include "explicit_diffusion.cuh"
#include "nesting.cuh"

using namespace wg;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

struct Dims {
  size_t m, u, v, w, s2, su, sv;  // element counts
};

Dims dims_of(const wrfgpu_step_params &p) {
  Dims d;
  const size_t nx = p.nx, ny = p.ny, nz = p.nz;
  d.m = nz * ny * nx;
  d.u = nz * ny * (nx + 1);
  d.v = nz * (ny + 1) * nx;
  d.w = (nz + 1) * ny * nx;
  d.s2 = ny * nx;
  d.su = ny * (nx + 1);
  d.sv = (ny + 1) * nx;
  return d;
}

// Bump allocator over the caller's workspace (256-byte aligned slices).
struct Carver {
  char *base;
  size_t off, cap;
  bool dry;
  double *take(size_t n) {
    off = (off + 255) & ~(size_t)255;
    double *p = dry ? nullptr : reinterpret_cast<double *>(base + off);
    off += n * sizeof(double);
    return p;
  }
};

struct Work {
  // 2-D
  double *mub, *mut, *muts0, *mu_work0, *muu, *muus, *muv, *muvs, *mu, *muts, *muave, *mudf, *phb0;
  double *rmsftx, *rmsfty, *rmsfux, *rmsfuy, *rmsfvx, *rmsfvy;  // map-factor reciprocals
  // mass
  double *alt_raw, *alt, *pb, *c2a, *qtot, *al_ls, *php_ls, *php, *t_tend, *theta_w, *t2ave, *p, *pm1, *al;
  double *s1, *s2, *ru, *rv, *dvdxi, *hdiv;
  LimFaces limf;  // limiter face fluxes (scale pass -> tendency pass)
  // per moisture species (set 0 = s1 / s2 / limf): the species are limited in
  // one scale-pass launch, each into its own scratch
  double *s1q[6], *s2q[6];
  LimFaces limq[6];
  double *qtend[6];
  // u / v faces
  double *u_tend, *u_w, *cqu, *u_target, *v_tend, *v_w, *cqv, *v_target;
  // w faces
  double *rom, *ww_spec, *rw_tend, *ph_tend, *cqw, *w_w, *ph_w, *pt1, *ww, *a, *alpha, *gamma;
  // intermediate states after stages 1 and 2
  StateW st[2];
  double *mu_tend_phys;  // physics: the stages' mu tendency (base + mu_tendf)
  double *xkmh;          // Smagorinsky eddy viscosity (mass cells)
  double *dz_part, *dz;  // constant K: per-row layer-depth sums and the mean
  // specified boundary cadence: the first stage's mu tendency (base + relax)
  double *mu_tend_s1;
};

bool is_moist(const wrfgpu_step_params &p) { return p.moist_adv_opt != 0; }
// the stage's second-order diffusion closures (operational_mode.py:2878-2960)
bool smag_on(const wrfgpu_step_params &p) { return p.diff_opt == 1 && p.km_opt == 4; }
bool constk_on(const wrfgpu_step_params &p) { return p.const_nu_m2_s > 0.0; }

void carve(const wrfgpu_step_params &p, Carver &c, Work &w) {
  const Dims d = dims_of(p);
  w.mub = c.take(d.s2); w.mut = c.take(d.s2); w.muts0 = c.take(d.s2); w.mu_work0 = c.take(d.s2);
  w.muu = c.take(d.su); w.muus = c.take(d.su); w.muv = c.take(d.sv); w.muvs = c.take(d.sv);
  w.mu = c.take(d.s2); w.muts = c.take(d.s2); w.muave = c.take(d.s2); w.mudf = c.take(d.s2);
  w.phb0 = c.take(d.s2);
  w.rmsftx = c.take(d.s2); w.rmsfty = c.take(d.s2); w.rmsfux = c.take(d.su); w.rmsfuy = c.take(d.su);
  w.rmsfvx = c.take(d.sv); w.rmsfvy = c.take(d.sv);
  w.alt_raw = c.take(d.m); w.alt = c.take(d.m); w.pb = c.take(d.m); w.c2a = c.take(d.m);
  w.qtot = c.take(d.m); w.al_ls = c.take(d.m); w.php_ls = c.take(d.m); w.php = c.take(d.m);
  w.t_tend = c.take(d.m); w.theta_w = c.take(d.m); w.t2ave = c.take(d.m); w.p = c.take(d.m);
  w.pm1 = c.take(d.m); w.al = c.take(d.m); w.ru = c.take(d.m); w.rv = c.take(d.m);
  w.dvdxi = c.take(d.m); w.hdiv = c.take(d.m);
  const bool lim = (p.scalar_adv_opt == 1 || p.scalar_adv_opt == 2 || p.moist_adv_opt == 1 || p.moist_adv_opt == 2);
  w.s1 = lim ? c.take(d.m) : nullptr;
  w.s2 = lim ? c.take(d.m) : nullptr;
  w.limf.lx = lim ? c.take(d.m) : nullptr; w.limf.ax = lim ? c.take(d.m) : nullptr;
  w.limf.ly = lim ? c.take(d.m) : nullptr; w.limf.ay = lim ? c.take(d.m) : nullptr;
  w.limf.lz = lim ? c.take(d.m) : nullptr; w.limf.az = lim ? c.take(d.m) : nullptr;
  const bool limq = p.moist_adv_opt == 1 || p.moist_adv_opt == 2;
  for (int q = 0; q < 6; ++q) {
    if (q == 0 || !limq) {
      w.s1q[q] = w.s1; w.s2q[q] = w.s2; w.limq[q] = w.limf;
      continue;
    }
    w.s1q[q] = c.take(d.m);
    w.s2q[q] = (p.moist_adv_opt == 2) ? c.take(d.m) : nullptr;  // the PD tendency reads s1 only
    w.limq[q].lx = c.take(d.m); w.limq[q].ax = c.take(d.m); w.limq[q].ly = c.take(d.m);
    w.limq[q].ay = c.take(d.m); w.limq[q].lz = c.take(d.m); w.limq[q].az = c.take(d.m);
  }
  for (int s = 0; s < 6; ++s) w.qtend[s] = is_moist(p) ? c.take(d.m) : nullptr;
  w.u_tend = c.take(d.u); w.u_w = c.take(d.u); w.cqu = c.take(d.u);
  w.v_tend = c.take(d.v); w.v_w = c.take(d.v); w.cqv = c.take(d.v);
  const bool bdy = p.run_boundary != 0;
  w.u_target = bdy ? c.take(d.u) : nullptr;
  w.v_target = bdy ? c.take(d.v) : nullptr;
  w.rom = c.take(d.w);
  const bool spec = p.run_boundary && !p.bc_ideal;
  w.ww_spec = spec ? c.take(d.w) : nullptr;
  w.rw_tend = c.take(d.w); w.ph_tend = c.take(d.w); w.cqw = c.take(d.w); w.w_w = c.take(d.w);
  w.ph_w = c.take(d.w); w.pt1 = c.take(d.w); w.ww = c.take(d.w);
  w.a = c.take(d.w); w.alpha = c.take(d.w); w.gamma = c.take(d.w);
  w.mu_tend_s1 = (spec && p.specified_bdy_cadence && p.force_geopotential) ? c.take(d.s2) : nullptr;
  w.mu_tend_phys = p.physics ? c.take(d.s2) : nullptr;
  w.xkmh = smag_on(p) ? c.take(d.m) : nullptr;
  w.dz_part = constk_on(p) ? c.take((size_t)p.ny) : nullptr;
  w.dz = constk_on(p) ? c.take(1) : nullptr;
  for (int s = 0; s < 2; ++s) {
    StateW &S = w.st[s];
    S.u = c.take(d.u); S.v = c.take(d.v); S.w = c.take(d.w); S.theta = c.take(d.m);
    S.p_total = c.take(d.m); S.p_pert = c.take(d.m); S.ph_total = c.take(d.w); S.ph_pert = c.take(d.w);
    S.mu_total = c.take(d.s2); S.mu_pert = c.take(d.s2);
    for (int q = 0; q < 6; ++q) S.q[q] = is_moist(p) ? c.take(d.m) : nullptr;
  }
}

StateR as_read(const StateW &s) {
  StateR r;
  r.u = s.u; r.v = s.v; r.w = s.w; r.theta = s.theta; r.p_total = s.p_total; r.p_pert = s.p_pert;
  r.ph_total = s.ph_total; r.ph_pert = s.ph_pert; r.mu_total = s.mu_total; r.mu_pert = s.mu_pert;
  for (int q = 0; q < 6; ++q) r.q[q] = s.q[q];
  return r;
}

Grid make_grid(const wrfgpu_step_params &p, const wrfgpu_metrics &m, const double *dn_host_top) {
  (void)dn_host_top;
  Grid g;
  g.nx = p.nx; g.ny = p.ny; g.nz = p.nz;
  g.dx = p.dx; g.dy = p.dy; g.rdx = 1.0 / p.dx; g.rdy = 1.0 / p.dy;
  g.c1h = m.c1h; g.c2h = m.c2h; g.c3h = m.c3h; g.c4h = m.c4h;
  g.c1f = m.c1f; g.c2f = m.c2f; g.c3f = m.c3f; g.c4f = m.c4f;
  g.dn = m.dn; g.dnw = m.dnw; g.rdn = m.rdn; g.rdnw = m.rdnw; g.fnm = m.fnm; g.fnp = m.fnp;
  g.msftx = m.msftx; g.msfty = m.msfty; g.msfux = m.msfux; g.msfuy = m.msfuy; g.msfvx = m.msfvx; g.msfvy = m.msfvy;
  g.f = m.f; g.e = m.e; g.sina = m.sina; g.cosa = m.cosa;
  g.cf1 = p.cf1; g.cf2 = p.cf2; g.cf3 = p.cf3; g.p_top = p.p_top;
  g.cfn = p.cfn; g.cfn1 = p.cfn1;
  return g;
}

// Specified boundary work targets (coupling/boundary_apply.py:729-781) for
// the normal momentum, from the time-interpolated strips.

// The targets are read by advance_uv only where its relax weight is non-zero:
// the relax_zone (<= nzone) columns (u) / rows (v) at each edge.  So only the
// nzone columns / rows at each edge are formed: index t in [0, 2 nzone) maps
// to t and x_len - 2 nzone + t (all columns when x_len <= 2 nzone, zero-padded
// targets outside the nzone bands there as before).
__device__ __forceinline__ int zone_index(int t, int len, int nzone) {
  return (len <= 2 * nzone || t < nzone) ? t : len - 2 * nzone + t;
}
__host__ __device__ inline int zone_extent(int len, int nzone) { return len <= 2 * nzone ? len : 2 * nzone; }

__global__ void k_bdy_target_u(Grid g, BdyLeaf b, const double *u_save, const double *muu, const double *muus,
                               int nzone, double *target) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int x_len = nx + 1;
  const int t_ = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (t_ >= zone_extent(x_len, nzone) || j >= ny) return;
  const int i = zone_index(t_, x_len, nzone);
  const size_t cu = ix3(k, j, i, ny, x_len);
  // last writer in the reference loop order: for b: W col b, then E col x_len-1-b
  int best = -1, side = 0;
  for (int bb = 0; bb < nzone; ++bb) {
    if (i == bb) { best = bb; side = 0; }
    if (i == x_len - 1 - bb) { best = bb; side = 1; }
  }
  double t = 0.0;
  if (best >= 0) {
    const size_t f2 = ix2(j, i, x_len);
    const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
    const double ms = c1 * ld(muus, f2) + c2, mc = c1 * ld(muu, f2) + c2;
    t = div_msf(strip_at(b, nz, side, best, k, j) * ms - ld(u_save, cu) * mc, g.msfuy, g.rmsfuy, f2);
  }
  target[cu] = t;
}

__global__ void k_bdy_target_v(Grid g, BdyLeaf b, const double *v_save, const double *muv, const double *muvs,
                               int nzone, double *target) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int y_len = ny + 1;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int t_ = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= nx || t_ >= zone_extent(y_len, nzone)) return;
  const int j = zone_index(t_, y_len, nzone);
  const size_t cv = ix3(k, j, i, y_len, nx);
  int best = -1, side = 2;
  for (int bb = 0; bb < nzone; ++bb) {
    if (j == bb) { best = bb; side = 2; }
    if (j == y_len - 1 - bb) { best = bb; side = 3; }
  }
  double t = 0.0;
  if (best >= 0) {
    const size_t f2 = ix2(j, i, nx);
    const double c1 = ld(g.c1h, k), c2 = ld(g.c2h, k);
    const double ms = c1 * ld(muvs, f2) + c2, mc = c1 * ld(muv, f2) + c2;
    t = div_msf(strip_at(b, nz, side, best, k, i) * ms - ld(v_save, cv) * mc, g.msfvx, g.rmsfvx, f2);
  }
  target[cv] = t;
}

// Correctly rounded map-factor reciprocals, once per step (index space
// (ny+1) x (nx+1) covers the mass, u-face and v-face 2-D shapes).
__global__ void k_recip_msf(Grid g, double *rtx, double *rty, double *rux, double *ruy, double *rvx, double *rvy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny;
  if (i < nx && j < ny) {
    const size_t c = ix2(j, i, nx);
    rtx[c] = 1.0 / ld(g.msftx, c);
    rty[c] = 1.0 / ld(g.msfty, c);
  }
  if (i <= nx && j < ny) {
    const size_t c = ix2(j, i, nx + 1);
    rux[c] = 1.0 / ld(g.msfux, c);
    ruy[c] = 1.0 / ld(g.msfuy, c);
  }
  if (i < nx && j <= ny) {
    const size_t c = ix2(j, i, nx);
    rvx[c] = 1.0 / ld(g.msfvx, c);
    rvy[c] = 1.0 / ld(g.msfvy, c);
  }
}

inline dim3 blk2() { return dim3(32, 4, 1); }
inline dim3 tblk() { return dim3(TSX, TSY, 1); }
inline dim3 tgrd(int nxx, int nyy, int nzz) { return dim3((nxx + TSX - 1) / TSX, (nyy + TSY - 1) / TSY, nzz); }
inline dim3 grd(int nxx, int nyy, int nzz) { return dim3((nxx + 31) / 32, (nyy + 3) / 4, nzz); }

int check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(WRFGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return WRFGPU_OK;
}

// ---------------------------------------------------------------------------
// Optional per-kernel timing: when enabled, every launch is bracketed by a
// pair of CUDA events (from a pool created at enable time) so a caller can
// read the device time of each kernel class over a region of steps.
// ---------------------------------------------------------------------------
struct ProfState {
  bool on = false;
  int cap = 0;
  int used = 0;
  std::vector<cudaEvent_t> ev;   // 2 per record
  std::vector<int> cls;
  cudaStream_t stream = nullptr;
};
ProfState g_prof;

const char *kClassNames[] = {"k_recip_msf", "k_mass2d", "k_transport", "k_diag", "k_uface", "k_vface", "k_mass", "k_lim_scale",
                             "k_lim_tend", "k_wface", "k_coef", "k_bdy_target_u", "k_bdy_target_v", "k_advance_uv",
                             "k_div_h", "k_column", "k_finish_u", "k_finish_v", "k_finish_col", "k_spec_relax",
                             "k_spec_w", "k_phys", "k_diff6", "k_constk", "k_smag"};
constexpr int kNumClasses = sizeof(kClassNames) / sizeof(kClassNames[0]);

int class_of(const char *name) {
  for (int c = 0; c < kNumClasses; ++c)
    if (std::strcmp(kClassNames[c], name) == 0) return c;
  return -1;
}

int g_pending_class = -1;

void prof_begin(const char *name, cudaStream_t s) {
  if (!g_prof.on) return;
  g_pending_class = -1;
  if (g_prof.used >= g_prof.cap) return;
  const int c = class_of(name);
  if (c < 0) return;
  cudaEventRecord(g_prof.ev[2 * g_prof.used], s);
  g_pending_class = c;
  g_prof.stream = s;
}

void prof_end(cudaStream_t s) {
  if (!g_prof.on || g_pending_class < 0) return;
  cudaEventRecord(g_prof.ev[2 * g_prof.used + 1], s);
  g_prof.cls[g_prof.used] = g_pending_class;
  g_prof.used += 1;
  g_pending_class = -1;
}

#define LAUNCH_CHECK(name)                      \
  do {                                          \
    prof_end(stream);                           \
    int _rc = check_launch(name);               \
    if (_rc != WRFGPU_OK) return _rc;           \
  } while (0)

#define PROF(name) prof_begin(name, stream)

}  // namespace

extern "C" {

const char *wrfgpu_last_error_string(void) { return g_last_error.c_str(); }

int wrfgpu_profile_enable(int enable, int max_records) {
  if (g_prof.on) {
    for (cudaEvent_t e : g_prof.ev) cudaEventDestroy(e);
    g_prof.ev.clear();
    g_prof.cls.clear();
    g_prof.on = false;
  }
  if (!enable) return WRFGPU_OK;
  if (max_records < 1) return fail(WRFGPU_ERR_BAD_SHAPE, "max_records must be >= 1");
  g_prof.ev.resize(2 * (size_t)max_records);
  g_prof.cls.assign(max_records, -1);
  for (auto &e : g_prof.ev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(WRFGPU_ERR_CUDA, "cudaEventCreate failed");
  g_prof.cap = max_records;
  g_prof.used = 0;
  g_prof.on = true;
  return WRFGPU_OK;
}

int wrfgpu_profile_read(double *total_ms, int *counts, int nclasses, int *dropped) {
  if (total_ms == nullptr || counts == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "output arrays are NULL");
  for (int c = 0; c < nclasses; ++c) {
    total_ms[c] = 0.0;
    counts[c] = 0;
  }
  if (!g_prof.on) return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "profiling is not enabled");
  if (g_prof.used > 0 && cudaEventSynchronize(g_prof.ev[2 * (g_prof.used - 1) + 1]) != cudaSuccess)
    return fail(WRFGPU_ERR_CUDA, "cudaEventSynchronize failed");
  for (int r = 0; r < g_prof.used; ++r) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, g_prof.ev[2 * r], g_prof.ev[2 * r + 1]) != cudaSuccess)
      return fail(WRFGPU_ERR_CUDA, "cudaEventElapsedTime failed");
    const int c = g_prof.cls[r];
    if (c >= 0 && c < nclasses) {
      total_ms[c] += ms;
      counts[c] += 1;
    }
  }
  if (dropped) *dropped = 0;
  g_prof.used = 0;
  return WRFGPU_OK;
}

int wrfgpu_profile_class_count(void) { return kNumClasses; }

const char *wrfgpu_profile_class_name(int c) { return (c >= 0 && c < kNumClasses) ? kClassNames[c] : ""; }

const char *wrfgpu_version(void) { return "wrfgpu-b200 0.1.0 (fp64 reference-order kernels, sm_100a)"; }

int wrfgpu_step_params_init(wrfgpu_step_params *p) {
  if (p == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "params is NULL");
  std::memset(p, 0, sizeof(*p));
  p->dt = 10.0;
  p->acoustic_substeps = 10;
  p->epssm = 0.1;
  p->top_lid = 0;
  p->w_damping = 0;
  p->damp_opt = 0;
  p->dampcoef = 0.0;
  p->zdamp = 5000.0;
  p->hypsometric_opt = 1;
  p->h_sca_adv_order = 2;
  p->scalar_adv_opt = 0;
  p->moist_adv_opt = 0;
  p->run_boundary = 0;
  p->bc_ideal = 1;
  p->spec_zone = 1;
  p->relax_zone = 4;
  p->update_cadence_s = 3600.0;
  p->normal_bdy_relax_strength = -1.0;
  p->force_geopotential = 1;
  p->diff_6th_factor = 0.12;  // operational_mode.py:492
  p->c_s = 0.25;              // operational_mode.py:482
  p->moist_cqw = 1;
  p->w_coriolis = 1;
  p->precision = WRFGPU_PRECISION_FP64;
  return WRFGPU_OK;
}

int wrfgpu_step_params_validate(const wrfgpu_step_params *p) {
  if (p == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "params is NULL");
  if (p->nz < 4) return fail(WRFGPU_ERR_BAD_SHAPE, "nz must be >= 4");
  if (p->nx < 1 || p->ny < 1) return fail(WRFGPU_ERR_BAD_SHAPE, "nx and ny must be >= 1");
  if ((double)(p->nz + 1) * (double)(p->ny + 1) * (double)(p->nx + 1) >= 2147483647.0)
    return fail(WRFGPU_ERR_BAD_SHAPE, "arrays of 2^31 or more elements are not supported (32-bit element offsets)");
  if (!(p->dx > 0.0) || !(p->dy > 0.0) || !(p->dt > 0.0)) return fail(WRFGPU_ERR_BAD_SHAPE, "dx, dy, dt must be > 0");
  if (p->acoustic_substeps < 1) return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "acoustic_substeps must be >= 1");
  if (p->hypsometric_opt != 1 && p->hypsometric_opt != 2)
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "hypsometric_opt must be 1 or 2");
  if (p->scalar_adv_opt < 0 || p->scalar_adv_opt > 2)
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "scalar_adv_opt must be 0, 1 or 2 (WENO options are not built)");
  if (p->moist_adv_opt < 0 || p->moist_adv_opt > 2)
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "moist_adv_opt must be 0, 1 or 2");
  const bool spec = p->run_boundary && !p->bc_ideal;
  if (spec && (p->nx < 3 || p->ny < 3)) return fail(WRFGPU_ERR_BAD_SHAPE, "specified boundaries need nx, ny >= 3");
  if (p->run_boundary && (p->spec_zone != 1 || p->relax_zone != 4))
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "boundary zones other than spec_zone=1, relax_zone=4 are not built");
  if (p->precision != WRFGPU_PRECISION_FP64 && p->precision != WRFGPU_PRECISION_MIXED)
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "unknown precision mode");
  if (p->march_levels != 0 && p->march_levels != 5 && p->march_levels != 10 && p->march_levels != 25)
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "march_levels must be 0, 5, 10 or 25");
  if (p->column_lanes != 0 && p->column_lanes != 8 && p->column_lanes != 13 && p->column_lanes != 16 &&
      p->column_lanes != 17)
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "column_lanes must be 0, 8, 13, 16 or 17");
  if (p->column_width != 0 && p->column_width != 1 && p->column_width != 16 && p->column_width != 32)
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "column_width must be 0, 1, 16 or 32");
  if (p->physics != 0 && p->physics != 1) return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "physics must be 0 or 1");
  if (p->diff_6th_opt && !(std::isfinite(p->diff_6th_factor) && p->diff_6th_factor >= 0.0))
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "diff_6th_factor must be finite and non-negative");
  if (p->diff_opt == 2 && (p->km_opt == 2 || p->km_opt == 3 || p->km_opt == 5))
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG,
                "diff_opt=2 with km_opt 2/3/5 (TKE / 3-D Smagorinsky closures) is not built");
  if (p->diff_opt == 1 && p->km_opt == 4 && !(std::isfinite(p->c_s) && p->c_s >= 0.0))
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "c_s must be finite and non-negative");
  if (!std::isfinite(p->const_nu_m2_s))
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "const_nu_m2_s must be finite");
  if (p->specified_adv_degrade != 0 && p->specified_adv_degrade != 1)
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "specified_adv_degrade must be 0 or 1");
  if (spec && p->specified_adv_degrade && p->force_geopotential && (p->nx < 7 || p->ny < 7))
    return fail(WRFGPU_ERR_BAD_SHAPE, "the specified advection degradation needs nx, ny >= 7");
  return WRFGPU_OK;
}

int wrfgpu_step_workspace_size(const wrfgpu_step_params *p, size_t *bytes) {
  if (p == nullptr || bytes == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "params/bytes is NULL");
  int rc = wrfgpu_step_params_validate(p);
  if (rc) return rc;
  Carver c{nullptr, 0, 0, true};
  Work w;
  carve(*p, c, w);
  *bytes = c.off + 256;
  return WRFGPU_OK;
}

int wrfgpu_step_launch_count(const wrfgpu_step_params *p, int *launches) {
  if (p == nullptr || launches == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "params/launches is NULL");
  int rc = wrfgpu_step_params_validate(p);
  if (rc) return rc;
  const int ns = p->acoustic_substeps;
  const int nsub[3] = {1, ns / 2 > 1 ? ns / 2 : 1, ns};
  const bool bdy = p->run_boundary != 0;
  int n = 1 + (p->physics ? 1 : 0);  // map-factor reciprocals [, the physics mu tendency]
  for (int s = 0; s < 3; ++s) {
    n += 8;  // mass2d, transport, diag, uface, vface, mass, wface, coef
    if (s == 2 && (p->scalar_adv_opt == 1 || p->scalar_adv_opt == 2)) n += 2;
    if (s == 2 && (p->moist_adv_opt == 1 || p->moist_adv_opt == 2)) n += 7;  // one scale pass, six tendency passes
    if (bdy) n += 2;
    n += 3 * nsub[s];  // advance_uv, div_h, column
    n += 3;  // finish u, v, col
    if (p->physics) n += 1;  // the physics merge of u, v, theta
    if (p->diff_6th_opt) n += 1;  // the 6th-order filter of u, v, w, theta
    if (constk_on(*p)) n += 3;    // constant K: layer-depth partials, mean, tendencies
    if (smag_on(*p)) n += 2;      // Smagorinsky: eddy viscosity, tendencies
    if (p->run_boundary && !p->bc_ideal && p->force_geopotential && p->specified_bdy_cadence) {
      n += (s == 0) ? 2 : 1;  // [first-stage mu tendency], relax tendencies
      n += nsub[s];           // zero-gradient w after every column launch
    }
    if (p->run_boundary && !p->bc_ideal && !p->force_geopotential && (p->nested_ph_relax || p->nested_w_relax))
      n += 1;  // the nested child's ph' / w relax tendencies
  }
  *launches = n;
  return WRFGPU_OK;
}

}  // extern "C"

namespace {

// The RK3 step.  The forecast lead is `lead_seconds` (host; NaN = no lead:
// boundary forcing off), or with `lead_dev` set a device-resident lead read
// by the kernels that interpolate boundary strips in time (`lead_seconds` is
// then only a non-NaN flag).
int rk3_step_impl(const wrfgpu_step_params *pp, const wrfgpu_metrics *mm, const wrfgpu_step_inputs *in,
                  const wrfgpu_step_outputs *out, double lead_seconds, const double *lead_dev, void *workspace,
                  size_t workspace_bytes, cudaStream_t stream) {
  if (pp == nullptr || mm == nullptr || in == nullptr || out == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "params/metrics/inputs/outputs is NULL");
  int rc = wrfgpu_step_params_validate(pp);
  if (rc) return rc;
  const wrfgpu_step_params &p = *pp;
  size_t need = 0;
  wrfgpu_step_workspace_size(pp, &need);
  if (workspace == nullptr || workspace_bytes < need)
    return fail(WRFGPU_ERR_WORKSPACE, "workspace is NULL or smaller than wrfgpu_step_workspace_size()");
  const double *req_in[] = {in->u, in->v, in->w, in->theta, in->p_total, in->p_perturbation, in->ph_total,
                            in->ph_perturbation, in->mu_total, in->mu_perturbation};
  for (const double *q : req_in)
    if (q == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "a required state input pointer is NULL");
  double *req_out[] = {out->u, out->v, out->w, out->theta, out->p_total, out->p_perturbation, out->ph_total,
                       out->ph_perturbation, out->mu_total, out->mu_perturbation};
  for (double *q : req_out)
    if (q == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "a required state output pointer is NULL");
  const bool moist = is_moist(p);
  const bool have_q = in->q[0] != nullptr;
  if (have_q)
    for (int s = 0; s < 6; ++s)
      if (in->q[s] == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "moisture inputs must be all NULL or all set");
  if (moist && !have_q) return fail(WRFGPU_ERR_NULL_POINTER, "moist_adv_opt != 0 needs the six moisture inputs");
  if (have_q)
    for (int s = 0; s < 6; ++s)
      if (out->q[s] == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "moisture outputs must be set when inputs are");
  const bool bdy_active = p.run_boundary && !std::isnan(lead_seconds);
  if (bdy_active && (in->u_bdy == nullptr || in->v_bdy == nullptr || in->bdy_ntime < 1 || in->bdy_width < 1 ||
                     in->bdy_side_len < (p.nx > p.ny ? p.nx + 1 : p.ny + 1)))
    return fail(WRFGPU_ERR_BAD_SHAPE, "run_boundary needs u_bdy/v_bdy strips (ntime, 4, width, nz, side_len)");
  // specified boundary cadence (operational_mode.py:2478-2492): on with the
  // flag, a specified domain and a forecast lead
  const bool cad = p.run_boundary && !p.bc_ideal && p.force_geopotential && p.specified_bdy_cadence &&
                   !std::isnan(lead_seconds);
  if (cad && (in->theta_bdy == nullptr || in->ph_bdy == nullptr || in->mu_bdy == nullptr || in->bdy_width < 5))
    return fail(WRFGPU_ERR_BAD_SHAPE,
                "specified_bdy_cadence needs theta_bdy/ph_bdy/mu_bdy strips (ntime, 4, width >= 5, nz | nz+1 | 1, side_len)");
  // the nested child's opt-in in-loop forcings (operational_mode.py:1906-1968):
  // a boundary domain without force_geopotential, with a forecast lead
  const bool nested = p.run_boundary && !p.bc_ideal && !p.force_geopotential && !std::isnan(lead_seconds);
  const bool nest_ph_relax = nested && p.nested_ph_relax, nest_w_relax = nested && p.nested_w_relax;
  const bool nest_ph_pin = nested && p.nested_ph_spec;
  if ((nest_ph_relax || nest_ph_pin) && (in->ph_bdy == nullptr || in->bdy_width < 5))
    return fail(WRFGPU_ERR_BAD_SHAPE, "nested_ph_relax / nested_ph_spec need the ph_bdy strip (width >= 5, nz+1 levels)");
  if (nest_w_relax && (in->w_bdy == nullptr || in->bdy_width < 5))
    return fail(WRFGPU_ERR_BAD_SHAPE, "nested_w_relax needs the w_bdy strip (width >= 5, nz+1 levels)");

  const Dims d = dims_of(p);
  Carver cv{reinterpret_cast<char *>(workspace), 0, workspace_bytes, false};
  Work w;
  carve(p, cv, w);
  Grid g = make_grid(p, *mm, nullptr);
  g.rmsftx = w.rmsftx; g.rmsfty = w.rmsfty; g.rmsfux = w.rmsfux; g.rmsfuy = w.rmsfuy;
  g.rmsfvx = w.rmsfvx; g.rmsfvy = w.rmsfvy;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const bool specified = p.run_boundary && !p.bc_ideal;
  const double dt = p.dt;
  const int ns = p.acoustic_substeps;
  const int kc = (p.march_levels == 5 || p.march_levels == 25) ? p.march_levels : MARCH_KC;
  const int lanes = (p.column_lanes > 0) ? p.column_lanes : COL_TY;
  const int cwidth = (p.column_width > 0) ? p.column_width : COL_DEFAULT_WIDTH;
  const bool col_stream = cwidth == 1;  // one thread per column (column_stream.cuh)
  const double dt_rk[3] = {dt / 3.0, 0.5 * dt, dt};
  const double dts_rk[3] = {dt / 3.0, dt / (double)ns, dt / (double)ns};
  const int nsub[3] = {1, ns / 2 > 1 ? ns / 2 : 1, ns};

  StateR origin;
  origin.u = in->u; origin.v = in->v; origin.w = in->w; origin.theta = in->theta;
  origin.p_total = in->p_total; origin.p_pert = in->p_perturbation;
  origin.ph_total = in->ph_total; origin.ph_pert = in->ph_perturbation;
  origin.mu_total = in->mu_total; origin.mu_pert = in->mu_perturbation;
  for (int s = 0; s < 6; ++s) origin.q[s] = in->q[s];
  StateW final_out;
  final_out.u = out->u; final_out.v = out->v; final_out.w = out->w; final_out.theta = out->theta;
  final_out.p_total = out->p_total; final_out.p_pert = out->p_perturbation;
  final_out.ph_total = out->ph_total; final_out.ph_pert = out->ph_perturbation;
  final_out.mu_total = out->mu_total; final_out.mu_pert = out->mu_perturbation;
  for (int s = 0; s < 6; ++s) final_out.q[s] = have_q ? out->q[s] : nullptr;

  // mudf carried across stages (operational_mode.py:2046)
  if (in->mudf != nullptr) {
    if (cudaMemcpyAsync(w.mudf, in->mudf, d.s2 * sizeof(double), cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      return fail(WRFGPU_ERR_CUDA, "mudf copy failed");
  } else if (cudaMemsetAsync(w.mudf, 0, d.s2 * sizeof(double), stream) != cudaSuccess) {
    return fail(WRFGPU_ERR_CUDA, "mudf clear failed");
  }

  const double eps1 = 1.0 + p.epssm;
  // a leaf with its time interpolation at the step's lead plus `off` seconds
  // (boundary_apply.py:329-345): resolved here, or by the kernels from the
  // device lead
  auto leaf_at_off = [&](const double *leaf, double off) {
    BdyLeaf b{leaf, in->bdy_ntime, in->bdy_width, in->bdy_side_len, 0, 0, 0.0, nullptr, 0.0, p.update_cadence_s};
    if (lead_dev != nullptr) {
      b.lead = lead_dev;
      b.lead_off = off;
    } else {
      leaf_time_weights(off == 0.0 ? lead_seconds : lead_seconds + off, p.update_cadence_s, in->bdy_ntime, b.lo,
                        b.hi, b.alpha);
    }
    return b;
  };
  BdyLeaf bl_u{}, bl_v{};
  if (bdy_active) {
    bl_u = leaf_at_off(in->u_bdy, 0.0);
    bl_v = leaf_at_off(in->v_bdy, 0.0);
  }
  RelaxArgs ra{};
  if (cad || nest_ph_relax || nest_w_relax) {
    // per-second weights as the reference forms them: (dt * fcx) / dt
    // (boundary_apply.py:666-688, 1031-1035)
    for (int b = 0; b < RELAX_B1; ++b) {
      ra.fcx[b] = 0.0;
      ra.gcx[b] = 0.0;
      if (b < RELAX_B0) continue;
      const double dtf = p.dt;
      const int loop = b + 1;
      const double num = (double)(p.spec_zone + p.relax_zone - loop), den = (double)(p.relax_zone - 1);
      double linear = num / den;
      linear = linear > 0.0 ? linear : 0.0;
      const double fcx = 0.1 / dtf * linear * 1.0;
      const double gcx = 1.0 / dtf / 50.0 * linear * 1.0;
      ra.fcx[b] = (dtf * fcx) / dtf;
      ra.gcx[b] = (dtf * gcx) / dtf;
    }
  }
  if (cad) {
    // relax_bdy_dry from the step-start state at the step-start lead
    // (boundary_apply.py:1148-1248)
    ra.u = in->u; ra.v = in->v; ra.theta = in->theta; ra.ph_pert = in->ph_perturbation;
    ra.mu_total = in->mu_total; ra.mu_pert = in->mu_perturbation;
    ra.lu = leaf_at_off(in->u_bdy, 0.0);
    ra.lv = leaf_at_off(in->v_bdy, 0.0);
    ra.lt = leaf_at_off(in->theta_bdy, 0.0);
    ra.lph = leaf_at_off(in->ph_bdy, 0.0);
    ra.lmu = leaf_at_off(in->mu_bdy, 0.0);
    ra.nfield = 5;
    const int cad_fields[5] = {RELAX_U, RELAX_V, RELAX_THETA, RELAX_PH, RELAX_MU};
    for (int f = 0; f < 5; ++f) ra.fields[f] = cad_fields[f];
  }

  PROF("k_recip_msf");
  k_recip_msf<<<grd(nx + 1, ny + 1, 1), blk2(), 0, stream>>>(g, w.rmsftx, w.rmsfty, w.rmsfux, w.rmsfuy, w.rmsfvx,
                                                             w.rmsfvy);
  LAUNCH_CHECK("k_recip_msf");
  // the stages' mu tendency: the base tendency, plus the physics mu_tendf
  const double *base_mu = in->base_mu;
  if (p.physics) {
    PROF("k_phys");
    k_phys_mu<<<grd(nx, ny, 1), blk2(), 0, stream>>>(g, in->base_mu, in->mu_tendf, w.mu_tend_phys);
    LAUNCH_CHECK("k_phys_mu");
    base_mu = w.mu_tend_phys;
  }
  PhysArgs phys{in->ru_tendf, in->rv_tendf, in->rw_tendf, in->t_tendf, in->mu_tendf, in->h_diabatic,
                in->phys_u_save, in->phys_v_save, in->phys_w_save, in->phys_t_save, 0};
  if (!p.physics) phys = PhysArgs{};

  // Advective-flux arithmetic: float64 (the reference's), or the mixed
  // variant's FP32 fluxes with float64 accumulation.
  const bool mixed = p.precision == WRFGPU_PRECISION_MIXED;
  // rhs_ph's order<=6 specified-boundary branch (core/rhs_ph.py:281-345)
  const bool ph_order6 = specified && p.h_sca_adv_order >= 4;
  // specified-boundary advection degradation (operational_mode.py:2464-2475,
  // 2494-2507; flux_advection.py:288-391): tiered faces, masked divergences,
  // a compile-time switch of the advection kernels
  const int deg = (specified && p.force_geopotential && p.specified_adv_degrade) ? 1 : 0;
  auto kUface = mixed ? (deg ? k_uface_tiled<float, true> : k_uface_tiled<float, false>)
                      : (deg ? k_uface_tiled<double, true> : k_uface_tiled<double, false>);
  auto kVface = mixed ? (deg ? k_vface_tiled<float, true> : k_vface_tiled<float, false>)
                      : (deg ? k_vface_tiled<double, true> : k_vface_tiled<double, false>);
#define WG_W(F, O) (deg ? k_wface_tiled<F, O, true> : k_wface_tiled<F, O, false>)
  auto kWface = mixed ? (ph_order6 ? WG_W(float, true) : WG_W(float, false))
                      : (ph_order6 ? WG_W(double, true) : WG_W(double, false));
#undef WG_W
  // marching kernels for the chosen chunk size (5, 10 or 25 levels)
  // (and for the specified degradation, a compile-time switch of their face fluxes)
#define WG_PICK_KC(tmpl, F, D) \
  (kc == 5 ? tmpl<F, 5, D> : kc == 25 ? tmpl<F, 25, D> : tmpl<F, 10, D>)
#define WG_PICK_KC_DEG(tmpl, F) (deg ? WG_PICK_KC(tmpl, F, true) : WG_PICK_KC(tmpl, F, false))
  auto kScalar = mixed ? WG_PICK_KC_DEG(k_scalar_adv_march, float) : WG_PICK_KC_DEG(k_scalar_adv_march, double);
  // the limiter's scale pass in each precision (the mixed variant stores its
  // face fluxes and scales as float32)
  auto kLimScaleF = WG_PICK_KC_DEG(k_lim_march, float);
  auto kLimScaleD = WG_PICK_KC_DEG(k_lim_march, double);
#undef WG_PICK_KC_DEG
#undef WG_PICK_KC

  StateR s = origin;
  for (int stage = 0; stage < 3; ++stage) {
    const int rk = stage + 1;
    const double dts = dts_rk[stage];
    StateW o = (stage == 2) ? final_out : w.st[stage];
    if (!moist && stage < 2) {
      for (int q = 0; q < 6; ++q) o.q[q] = nullptr;  // moisture passes through untouched
    }
    Mass2D m2{w.mub, w.mut, w.muts0, w.mu_work0, w.muu, w.muus, w.muv, w.muvs, w.mu, w.muts, w.muave};
    PROF("k_mass2d");
    k_mass2d<<<grd(nx + 1, ny + 1, 1), blk2(), 0, stream>>>(g, s, origin.mu_pert, rk, m2);
    LAUNCH_CHECK("k_mass2d");
    PROF("k_transport");
    k_transport_tiled<<<dim3((nx + 31) / 32, ny, 1), dim3(32, 8, 1), transport_smem_bytes(nz), stream>>>(
        g, s.u, s.v, s.mu_total, w.ru, w.rv, w.rom, specified ? w.ww_spec : nullptr);
    LAUNCH_CHECK("k_transport");
    Diag dg{w.alt_raw, w.alt, w.pb, w.c2a, w.qtot, w.al_ls, w.php_ls, w.php};
    PROF("k_diag");
    k_diag<<<grd(nx, ny, nz), blk2(), 0, stream>>>(g, s, p.hypsometric_opt, dg);
    LAUNCH_CHECK("k_diag");
    UFaceOut uo{w.u_tend, w.u_w, w.cqu};
    PROF("k_uface");
    kUface<<<tgrd(nx + 1, ny, nz), tblk(), 0, stream>>>(g, s, origin, w.ru, w.rv, w.rom, dg, w.muu, w.muus,
                                                               in->base_u, p.top_lid, p.run_boundary, uo);
    LAUNCH_CHECK("k_uface");
    VFaceOut vo{w.v_tend, w.v_w, w.cqv};
    PROF("k_vface");
    kVface<<<tgrd(nx, ny + 1, nz), tblk(), 0, stream>>>(g, s, origin, w.ru, w.rv, w.rom, dg, w.muv, w.muvs,
                                                               in->base_v, p.top_lid, p.run_boundary, vo);
    LAUNCH_CHECK("k_vface");
    const bool lim_theta = (rk == 3) && (p.scalar_adv_opt == 1 || p.scalar_adv_opt == 2);
    const bool lim_moist = moist && (rk == 3) && (p.moist_adv_opt == 1 || p.moist_adv_opt == 2);
    MassOut mo;
    mo.t_tend = w.t_tend;
    mo.theta_w = w.theta_w;
    for (int q = 0; q < 6; ++q) {
      mo.q_tend[q] = w.qtend[q];
      mo.q_tend32[q] = reinterpret_cast<float *>(w.qtend[q]);
    }
    PROF("k_mass");
    {
      const int nfields = 1 + ((moist && !lim_moist) ? 6 : 0);
      const int nchunk = march_nchunk(nz, kc);
      kScalar<<<tgrd(nx, ny, nfields * nchunk), tblk(), 0, stream>>>(
          g, s, origin, w.ru, w.rv, w.rom, w.mut, w.muts0, in->base_theta, lim_theta ? 0 : 1, nfields, mo);
    }
    LAUNCH_CHECK("k_mass");
    if (lim_theta || lim_moist) {
      LimArgs la;
      la.ru = w.ru; la.rv = w.rv; la.rom = w.rom; la.mut = s.mu_total; la.mu_old = origin.mu_total; la.dt = dt;
      la.deg = deg;
      set_lim_constants(la, g.rdx, g.rdy);
      // float32 views of the same scratch for the mixed variant
      auto f32 = [](const LimFaces &f) {
        return LimFacesT<float>{reinterpret_cast<float *>(f.lx), reinterpret_cast<float *>(f.ax),
                                reinterpret_cast<float *>(f.ly), reinterpret_cast<float *>(f.ay),
                                reinterpret_cast<float *>(f.lz), reinterpret_cast<float *>(f.az)};
      };
      const LimFacesT<float> limf32 = f32(w.limf);
      float *s1f = reinterpret_cast<float *>(w.s1), *s2f = reinterpret_cast<float *>(w.s2);
      // one scale-pass launch over n fields (theta alone, or the six species),
      // each into its own scratch set
      auto scale_pass = [&](int n, const double *const *fld, const double *const *fld_old, int set0) {
        const dim3 lim_grid(((nx + TSX - 1) / TSX) * n, (ny + TSY - 1) / TSY, march_nchunk(nz, kc));
        if (mixed) {
          LimBatch<float> lb{};
          lb.n = n;
          for (int t = 0; t < n; ++t) {
            lb.field[t] = fld[t]; lb.field_old[t] = fld_old[t];
            lb.s1[t] = reinterpret_cast<float *>(w.s1q[set0 + t]);
            lb.s2[t] = reinterpret_cast<float *>(w.s2q[set0 + t]);
            lb.fo[t] = f32(w.limq[set0 + t]);
          }
          kLimScaleF<<<lim_grid, tblk(), 0, stream>>>(g, la, lb);
        } else {
          LimBatch<double> lb{};
          lb.n = n;
          for (int t = 0; t < n; ++t) {
            lb.field[t] = fld[t]; lb.field_old[t] = fld_old[t];
            lb.s1[t] = w.s1q[set0 + t]; lb.s2[t] = w.s2q[set0 + t]; lb.fo[t] = w.limq[set0 + t];
          }
          kLimScaleD<<<lim_grid, tblk(), 0, stream>>>(g, la, lb);
        }
      };
      if (lim_theta) {
        la.opt = p.scalar_adv_opt;
        la.offset = T0;
        PROF("k_lim_scale");
        const double *th[1] = {s.theta}, *th0[1] = {origin.theta};
        scale_pass(1, th, th0, 0);
        LAUNCH_CHECK("k_lim_scale");
        PROF("k_lim_tend");
        // theta's tendency stays float64 (the acoustic loop reads it)
        if (mixed)
          k_lim_tend_faces<float, double><<<grd(nx, ny, nz), blk2(), 0, stream>>>(g, la, limf32, s1f, s2f,
                                                                                in->base_theta, s.mu_total, w.t_tend);
        else
          k_lim_tend_faces<double, double><<<grd(nx, ny, nz), blk2(), 0, stream>>>(g, la, w.limf, w.s1, w.s2,
                                                                                 in->base_theta, s.mu_total,
                                                                                 w.t_tend);
        LAUNCH_CHECK("k_lim_tend");
      }
      if (lim_moist) {
        la.opt = p.moist_adv_opt;
        la.offset = 0.0;
        PROF("k_lim_scale");
        scale_pass(6, s.q, origin.q, 0);
        LAUNCH_CHECK("k_lim_scale");
        for (int q = 0; q < 6; ++q) {
          PROF("k_lim_tend");
          if (mixed)
            k_lim_tend_faces<float, float><<<grd(nx, ny, nz), blk2(), 0, stream>>>(
                g, la, f32(w.limq[q]), reinterpret_cast<float *>(w.s1q[q]), reinterpret_cast<float *>(w.s2q[q]),
                nullptr, s.mu_total, reinterpret_cast<float *>(w.qtend[q]));
          else
            k_lim_tend_faces<double, double><<<grd(nx, ny, nz), blk2(), 0, stream>>>(
                g, la, w.limq[q], w.s1q[q], w.s2q[q], nullptr, s.mu_total, w.qtend[q]);
          LAUNCH_CHECK("k_lim_tend");
        }
      }
    }
    const double *ww_stage = specified ? w.ww_spec : w.rom;
    WFaceOut wo{w.rw_tend, w.ph_tend, w.cqw, w.w_w, w.ph_w, w.pt1, w.ww, w.phb0};
    PROF("k_wface");
    kWface<<<tgrd(nx, ny, nz + 1), tblk(), 0, stream>>>(g, s, origin, w.ru, w.rv, w.rom, ww_stage, w.qtot,
                                                               w.mub, w.mut, w.muts0, w.muu, w.muv, in->base_w,
                                                               p.top_lid, p.moist_cqw, p.w_coriolis, wo,
                                                               PhysW{phys.rw_tendf, phys.w_save, stage == 0 ? 1 : 0});
    LAUNCH_CHECK("k_wface");
    const double x = 0.5 * dts * G * eps1;
    const double cof = x * x;
    CoefOut co{w.a, w.alpha, w.gamma, w.p, w.pm1, w.al, w.t2ave};
    const size_t coef_smem = coef_smem_bytes(nz);
    if (stage == 0 && cudaFuncSetAttribute(k_coef, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coef_smem) !=
                          cudaSuccess)
      return fail(WRFGPU_ERR_CUDA, "cannot reserve shared memory for k_coef (nz too large)");
    PROF("k_coef");
    k_coef<<<dim3((nx + 31) / 32, ny, 1), dim3(32, COEF_TY, 1), coef_smem, stream>>>(
        g, w.mut, w.muts0, w.mu_work0, w.c2a, w.cqw, w.alt, w.theta_w, w.ph_w, origin.theta, cof, p.top_lid, co);
    LAUNCH_CHECK("k_coef");

    if (p.diff_6th_opt) {
      // the 6th-order filter of the stage state into its coupled tendencies
      // (operational_mode.py:2870-2876), ahead of the physics merge
      Diff6Args da{s.u, s.v, s.w, s.theta, s.mu_total, w.u_tend, w.v_tend, w.rw_tend, w.t_tend,
                   p.diff_6th_factor * 0.015625 / (2.0 * p.dt)};
      PROF("k_diff6");
      k_diff6<<<dim3((nx + 1 + D6_TX - 1) / D6_TX, (ny + 1 + D6_TY - 1) / D6_TY, (nz + 1 + D6_KC - 1) / D6_KC),
                dim3(D6_TX, D6_TY, 1), 0, stream>>>(g, da);
      LAUNCH_CHECK("k_diff6");
    }
    if (constk_on(p) || smag_on(p)) {
      DiffArgs xa{s.u, s.v, s.w, s.theta, s.mu_total, w.u_tend, w.v_tend, w.rw_tend, w.t_tend,
                  w.xkmh, p.c_s, p.const_nu_m2_s, w.dz};
      const dim3 agrid = grd(nx + 1, ny + 1, nz + 1);
      if (constk_on(p)) {
        // constant K (operational_mode.py:2878-2929), the stage's mean layer depth first
        PROF("k_constk");
        k_dz_partial<<<ny, DZ_THREADS, 0, stream>>>(g, s.ph_total, w.dz_part);
        LAUNCH_CHECK("k_dz_partial");
        PROF("k_constk");
        k_dz_final<<<1, 32, 0, stream>>>(g, w.dz_part, w.dz);
        LAUNCH_CHECK("k_dz_final");
        PROF("k_constk");
        k_constk_apply<<<agrid, blk2(), 0, stream>>>(g, xa);
        LAUNCH_CHECK("k_constk_apply");
      }
      if (smag_on(p)) {
        // 2-D Smagorinsky (operational_mode.py:2946-2960)
        PROF("k_smag");
        k_smag_km<<<grd(nx, ny, nz), blk2(), 0, stream>>>(g, xa, w.xkmh);
        LAUNCH_CHECK("k_smag_km");
        PROF("k_smag");
        k_smag_apply<<<agrid, blk2(), 0, stream>>>(g, xa);
        LAUNCH_CHECK("k_smag_apply");
      }
    }
    if (p.physics) {
      // rk_addtend_dry: the physics tendencies into this stage's u, v, theta (w: in k_wface)
      PhysArgs ps = phys;
      ps.rk1 = (stage == 0) ? 1 : 0;
      PROF("k_phys");
      k_phys_merge<<<grd(nx + 1, ny + 1, nz), blk2(), 0, stream>>>(g, ps, s.mu_total, w.u_tend, w.v_tend, w.t_tend);
      LAUNCH_CHECK("k_phys_merge");
    }
    if (cad) {
      // relax tendencies into this stage's u, v, theta and ph' tendencies, and
      // (first stage only) the mu' tendency (operational_mode.py:1994-1995, 3085-3092)
      if (stage == 0) {
        PROF("k_spec_relax");
        k_mu_tend_init<<<grd(nx, ny, 1), blk2(), 0, stream>>>(g, base_mu, w.mu_tend_s1);
        LAUNCH_CHECK("k_mu_tend_init");
      }
      RelaxArgs rs = ra;
      rs.u_tend = w.u_tend; rs.v_tend = w.v_tend; rs.t_tend = w.t_tend; rs.ph_tend = w.ph_tend;
      rs.mu_tend = (stage == 0) ? w.mu_tend_s1 : nullptr;
      const int ring_len = 2 * (nx + 1) + 2 * (ny + 1);
      PROF("k_spec_relax");
      k_spec_relax_add<<<dim3((ring_len + 127) / 128, RELAX_B1 - RELAX_B0, rs.nfield * (nz + 1)), 128, 0, stream>>>(
          g, rs);
      LAUNCH_CHECK("k_spec_relax_add");
    }
    if (nest_ph_relax || nest_w_relax) {
      // the nested child's relax-zone ph' / w tendencies from the stage state,
      // coupled with the stage mass, leaves at the step's lead, into this
      // stage's ph and rw tendencies (operational_mode.py:1925-1959)
      RelaxArgs rn = ra;
      rn.ph_pert = s.ph_pert; rn.w = s.w; rn.mu_total = w.mut;
      rn.ph_tend = w.ph_tend; rn.rw_tend = w.rw_tend;
      rn.nfield = 0;
      if (nest_ph_relax) {
        rn.lph = leaf_at_off(in->ph_bdy, 0.0);
        rn.fields[rn.nfield++] = RELAX_PH;
      }
      if (nest_w_relax) {
        rn.lw = leaf_at_off(in->w_bdy, 0.0);
        rn.fields[rn.nfield++] = RELAX_W;
      }
      const int ring_len = 2 * (nx + 1) + 2 * (ny + 1);
      PROF("k_spec_relax");
      k_spec_relax_add<<<dim3((ring_len + 127) / 128, RELAX_B1 - RELAX_B0, rn.nfield * (nz + 1)), 128, 0, stream>>>(
          g, rn);
      LAUNCH_CHECK("k_spec_relax_add");
    }
    // the ring-0 pins interpolate the strips at the stage-end lead, lead + dt_rk[stage]

    BdyArgs ba{};
    ba.active = bdy_active ? 1 : 0;
    ba.cad = cad ? 1 : 0;
    if (cad) {
      ba.cad_u = leaf_at_off(in->u_bdy, dt_rk[stage]);
      ba.cad_v = leaf_at_off(in->v_bdy, dt_rk[stage]);
    }
    if (bdy_active) {
      const int nzone = p.spec_zone + p.relax_zone;
      PROF("k_bdy_target_u");
      k_bdy_target_u<<<grd(zone_extent(nx + 1, nzone), ny, nz), blk2(), 0, stream>>>(g, bl_u, s.u, w.muu, w.muus,
                                                                                     nzone, w.u_target);
      LAUNCH_CHECK("k_bdy_target_u");
      PROF("k_bdy_target_v");
      k_bdy_target_v<<<grd(nx, zone_extent(ny + 1, nzone), nz), blk2(), 0, stream>>>(g, bl_v, s.v, w.muv, w.muvs,
                                                                                     nzone, w.v_target);
      LAUNCH_CHECK("k_bdy_target_v");
      const double strength = (p.normal_bdy_relax_strength < 0.0) ? 20.0 : p.normal_bdy_relax_strength;
      ba.u_target = w.u_target;
      ba.v_target = w.v_target;
      ba.sub_ratio = strength * (dt != 0.0 ? dts / dt : 0.0);
      ba.spec_zone = 1;  // apply_normal_bdy_work uses DEFAULT_BOUNDARY_CONFIG widths
      ba.relax_zone = 4;
      set_bdy_weights(ba);
    }

    Acoustic A;
    A.u = w.u_w; A.v = w.v_w; A.w = w.w_w; A.ph = w.ph_w; A.theta_w = w.theta_w; A.t2ave = w.t2ave;
    A.p = w.p; A.pm1 = w.pm1; A.al = w.al; A.ww = w.ww;
    A.mu = w.mu; A.muts = w.muts; A.muave = w.muave; A.mudf = w.mudf;
    A.u_tend = w.u_tend; A.v_tend = w.v_tend; A.t_tend = w.t_tend; A.rw_tend = w.rw_tend; A.ph_tend = w.ph_tend;
    A.alt = w.alt; A.pb = w.pb; A.c2a = w.c2a; A.cqu = w.cqu; A.cqv = w.cqv; A.cqw = w.cqw; A.php = w.php;
    A.pt1 = w.pt1; A.a = w.a; A.alpha = w.alpha; A.gamma = w.gamma; A.ww_1 = ww_stage;
    A.mut = w.mut; A.muu = w.muu; A.muv = w.muv; A.muus = w.muus; A.muvs = w.muvs;
    A.mu_tend = (cad && stage == 0) ? w.mu_tend_s1 : base_mu;
    A.u_1 = s.u; A.v_1 = s.v; A.w_save = s.w; A.theta_s = s.theta; A.phb0 = w.phb0;
    ColArgs ca{};
    ca.dts = dts; ca.epssm = p.epssm; ca.specified = specified ? 1 : 0; ca.top_lid = p.top_lid;
    ca.w_damping = p.w_damping; ca.damp_opt = p.damp_opt; ca.dampcoef = p.dampcoef; ca.zdamp = p.zdamp;
    ca.rzdamp = (p.zdamp != 0.0 && std::isfinite(1.0 / p.zdamp)) ? 1.0 / p.zdamp : 0.0;
    ca.cad = cad ? 1 : 0;
    if (cad) {
      ca.cad_mu = leaf_at_off(in->mu_bdy, dt_rk[stage]);
      ca.cad_th = leaf_at_off(in->theta_bdy, dt_rk[stage]);
      ca.mub = w.mub;
    }
    ca.ph_pin = (cad || nest_ph_pin) ? 1 : 0;
    if (ca.ph_pin) {
      // the cadence pins to the stage-end lead, the nested child to the step's lead
      ca.cad_ph = leaf_at_off(in->ph_bdy, cad ? dt_rk[stage] : 0.0);
      ca.ph_save = s.ph_pert;
    }
    const size_t col_smem = col_stream ? column_stream_smem_bytes(nz) : column_tiled_smem_bytes(nz, cwidth);
    // the ring-0 pins are compiled into their own instantiations
    const bool pins = cad || nest_ph_pin;
#define WG_COL(TX, TY) (pins ? k_column_tiled<TX, TY, true> : k_column_tiled<TX, TY, false>)
    auto kColumn = col_stream ? (pins ? k_column_stream<true> : k_column_stream<false>)
                   : (cwidth == 16) ? ((lanes == 8)    ? WG_COL(16, 8)
                                       : (lanes == 16) ? WG_COL(16, 16)
                                       : (lanes == 17) ? WG_COL(16, 17)
                                                       : WG_COL(16, 13))
                                    : ((lanes == 8)    ? WG_COL(32, 8)
                                       : (lanes == 16) ? WG_COL(32, 16)
                                       : (lanes == 17) ? WG_COL(32, 17)
                                                       : WG_COL(32, 13));
#undef WG_COL
    const dim3 col_grid = col_stream ? dim3((nx + 31) / 32, (ny + CS_WARPS - 1) / CS_WARPS, 1)
                                     : dim3((nx + cwidth - 1) / cwidth, ny, 1);
    const dim3 col_block = col_stream ? dim3(32, CS_WARPS, 1) : dim3(cwidth, lanes, 1);
    auto kAdvanceUV = cad ? k_advance_uv<true> : k_advance_uv<false>;
    if (stage == 0 && cudaFuncSetAttribute(kColumn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem) !=
                          cudaSuccess)
      return fail(WRFGPU_ERR_CUDA, "cannot reserve shared memory for k_column_tiled (nz too large)");
    for (int it = 0; it < nsub[stage]; ++it) {
      PROF("k_advance_uv");
      kAdvanceUV<<<grd(nx + 1, ny + 1, (nz + UV_KC - 1) / UV_KC), blk2(), 0, stream>>>(g, A, dts, p.top_lid,
                                                                                              ba);
      LAUNCH_CHECK("k_advance_uv");
      PROF("k_div_h");
      k_div_h<<<grd(nx, ny, nz), blk2(), 0, stream>>>(g, A, specified ? 1 : 0, w.dvdxi, w.hdiv);
      LAUNCH_CHECK("k_div_h");
      PROF("k_column");
      kColumn<<<col_grid, col_block, col_smem, stream>>>(g, A, ca, w.dvdxi, w.hdiv);
      LAUNCH_CHECK("k_column");
      if (cad) {
        PROF("k_spec_w");
        const int ring0 = 2 * nx + 2 * (ny - 2);
        k_spec_w_zero_grad<<<dim3((ring0 + 127) / 128, nz + 1, 1), 128, 0, stream>>>(g, w.w_w, s.w, w.mut, w.muts);
        LAUNCH_CHECK("k_spec_w_zero_grad");
      }
    }

    PROF("k_finish_u");
    k_finish_u<<<grd(nx + 1, ny, nz), blk2(), 0, stream>>>(g, w.u_w, s.u, w.muu, w.muus, o.u);
    LAUNCH_CHECK("k_finish_u");
    PROF("k_finish_v");
    k_finish_v<<<grd(nx, ny + 1, nz), blk2(), 0, stream>>>(g, w.v_w, s.v, w.muv, w.muvs, o.v);
    LAUNCH_CHECK("k_finish_v");
    FinishArgs fa;
    fa.w_w = w.w_w; fa.ph_w = w.ph_w; fa.theta_w = w.theta_w; fa.p_ac = w.p; fa.mu_ac = w.mu; fa.muts_ac = w.muts;
    fa.t2ave = w.t2ave; fa.ww_ac = w.ww; fa.mut = w.mut; fa.ww_stage = ww_stage;
    for (int q = 0; q < 6; ++q) {
      fa.q_tend[q] = w.qtend[q];
      fa.q_tend32[q] = reinterpret_cast<const float *>(w.qtend[q]);
    }
    fa.q32 = mixed ? 1 : 0;
    fa.dt_rk = dt_rk[stage];
    fa.hyps = p.hypsometric_opt;
    fa.moist = moist ? 1 : 0;
    fa.t_2ave_out = (stage == 2) ? out->t_2ave : nullptr;
    fa.ww_out = (stage == 2) ? out->ww : nullptr;
    fa.t_save_out = (stage == 2) ? out->t_save : nullptr;
    PROF("k_finish_col");
    k_finish_cells<<<grd(nx, ny, nz + 1), blk2(), 0, stream>>>(g, s, origin, fa, o);
    LAUNCH_CHECK("k_finish_col");

    if (stage == 2) {
      struct Cp { double *dst; const double *src; size_t n; } cps[] = {
          {out->mudf, w.mudf, d.s2},       {out->muave, w.muave, d.s2},   {out->muts, w.muts, d.s2},
          {out->ph_tend, w.ph_tend, d.w},  {out->u_save, s.u, d.u},       {out->v_save, s.v, d.v},
          {out->w_save, s.w, d.w},         {out->ph_save, s.ph_pert, d.w}, {out->mu_save, s.mu_pert, d.s2},
          {out->ww_save, ww_stage, d.w}};
      for (const Cp &c : cps) {
        if (c.dst == nullptr) continue;
        if (cudaMemcpyAsync(c.dst, c.src, c.n * sizeof(double), cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
          return fail(WRFGPU_ERR_CUDA, "carry output copy failed");
      }
    }
    StateR next = as_read(o);
    if (!moist) {
      for (int q = 0; q < 6; ++q) next.q[q] = (stage == 2) ? next.q[q] : origin.q[q];
    }
    s = next;
  }
  g_last_error.clear();
  return WRFGPU_OK;
}

}  // namespace

extern "C" {

int wrfgpu_rk3_step(const wrfgpu_step_params *pp, const wrfgpu_metrics *mm, const wrfgpu_step_inputs *in,
                    const wrfgpu_step_outputs *out, double lead_seconds, void *workspace, size_t workspace_bytes,
                    cudaStream_t stream) {
  return rk3_step_impl(pp, mm, in, out, lead_seconds, nullptr, workspace, workspace_bytes, stream);
}

int wrfgpu_rk3_step_device_lead(const wrfgpu_step_params *pp, const wrfgpu_metrics *mm,
                                const wrfgpu_step_inputs *in, const wrfgpu_step_outputs *out,
                                const double *lead_seconds_dev, void *workspace, size_t workspace_bytes,
                                cudaStream_t stream) {
  if (lead_seconds_dev == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "lead_seconds_dev is NULL");
  return rk3_step_impl(pp, mm, in, out, 0.0, lead_seconds_dev, workspace, workspace_bytes, stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Step with a library-held workspace, for callers that cannot allocate device
// memory.  The array lives in this module on every GPU that loads it; its
// device address is looked up once per GPU (with that GPU current) and then
// reused.  No cudaMalloc/cudaFree or allocating library routine is called.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_static_workspace[WRFGPU_STATIC_WORKSPACE_BYTES];

namespace {
constexpr int kMaxStaticDevices = 64;
std::mutex g_static_ws_mutex;
// Device address of the array per device ordinal, looked up on the first call
// and kept for the life of the process.  It belongs to the device context that
// was current then: after cudaDeviceReset (or anything else that destroys and
// recreates the primary context) the module is loaded again and this cached
// address is stale, so a process that resets a device must not call the
// static-workspace step on it afterwards.
void *g_static_ws_addr[kMaxStaticDevices] = {};
}  // namespace

extern "C" int wrfgpu_rk3_step_static_workspace(const wrfgpu_step_params *pp, const wrfgpu_metrics *mm,
                                                const wrfgpu_step_inputs *in, const wrfgpu_step_outputs *out,
                                                double lead_seconds, cudaStream_t stream) {
  if (pp == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "params is NULL");
  int rc = wrfgpu_step_params_validate(pp);
  if (rc) return rc;
  size_t need = 0;
  rc = wrfgpu_step_workspace_size(pp, &need);
  if (rc) return rc;
  if (need > WRFGPU_STATIC_WORKSPACE_BYTES)
    return fail(WRFGPU_ERR_WORKSPACE,
                "grid needs " + std::to_string(need) + " workspace bytes but the library-held workspace has " +
                    std::to_string((size_t)WRFGPU_STATIC_WORKSPACE_BYTES) +
                    "; use wrfgpu_rk3_step with a caller workspace for this grid");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(WRFGPU_ERR_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxStaticDevices)
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "device ordinal out of range for the library-held workspace");
  void *ws = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_static_ws_mutex);
    if (g_static_ws_addr[dev] == nullptr) {
      void *addr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&addr, g_static_workspace);
      if (e != cudaSuccess || addr == nullptr)
        return fail(WRFGPU_ERR_CUDA, std::string("cudaGetSymbolAddress of the library-held workspace failed: ") +
                                         cudaGetErrorString(e));
      g_static_ws_addr[dev] = addr;
    }
    ws = g_static_ws_addr[dev];
  }
  return wrfgpu_rk3_step(pp, mm, in, out, lead_seconds, ws, WRFGPU_STATIC_WORKSPACE_BYTES, stream);
}

// ---------------------------------------------------------------------------
// Batched step: members forked onto a per-device pool of library streams.
// ---------------------------------------------------------------------------
namespace {
#ifndef WG_POOL_STREAMS
#define WG_POOL_STREAMS 8
#endif
constexpr int kPoolStreams = WG_POOL_STREAMS;
constexpr int kMaxPoolDevices = 64;
struct StreamPool {
  cudaStream_t s[kPoolStreams];
  cudaEvent_t fork;
  cudaEvent_t join[kPoolStreams];
  bool ready = false;
};
std::mutex g_pool_mutex;
StreamPool g_pools[kMaxPoolDevices];

int pool_for_current_device(StreamPool **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(WRFGPU_ERR_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxPoolDevices) return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  StreamPool &p = g_pools[dev];
  if (!p.ready) {
    if (cudaEventCreateWithFlags(&p.fork, cudaEventDisableTiming) != cudaSuccess)
      return fail(WRFGPU_ERR_CUDA, "cannot create the batch fork event");
    for (int k = 0; k < kPoolStreams; ++k) {
      if (cudaStreamCreateWithFlags(&p.s[k], cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&p.join[k], cudaEventDisableTiming) != cudaSuccess)
        return fail(WRFGPU_ERR_CUDA, "cannot create the batch stream pool");
    }
    p.ready = true;
  }
  *out = &p;
  return WRFGPU_OK;
}
}  // namespace

extern "C" int wrfgpu_rk3_step_batched(int n, const wrfgpu_step_params *params, const wrfgpu_metrics *metrics,
                                       const wrfgpu_step_inputs *in, const wrfgpu_step_outputs *out,
                                       const double *lead_seconds, void *const *workspace,
                                       const size_t *workspace_bytes, cudaStream_t stream) {
  if (n < 0) return fail(WRFGPU_ERR_BAD_SHAPE, "n must be >= 0");
  if (n == 0) return WRFGPU_OK;
  if (params == nullptr || metrics == nullptr || in == nullptr || out == nullptr || lead_seconds == nullptr ||
      workspace == nullptr || workspace_bytes == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "a batch array is NULL");
  // validate every member before enqueueing anything
  for (int m = 0; m < n; ++m) {
    int rc = wrfgpu_step_params_validate(&params[m]);
    if (rc) return rc;
    size_t need = 0;
    wrfgpu_step_workspace_size(&params[m], &need);
    if (workspace[m] == nullptr || workspace_bytes[m] < need)
      return fail(WRFGPU_ERR_WORKSPACE, "member " + std::to_string(m) + ": workspace is NULL or too small");
  }
  if (n == 1) return wrfgpu_rk3_step(&params[0], &metrics[0], &in[0], &out[0], lead_seconds[0], workspace[0],
                                     workspace_bytes[0], stream);
  StreamPool *pool = nullptr;
  int rc = pool_for_current_device(&pool);
  if (rc) return rc;
  const int used = n < kPoolStreams ? n : kPoolStreams;
  if (cudaEventRecord(pool->fork, stream) != cudaSuccess) return fail(WRFGPU_ERR_CUDA, "fork record failed");
  for (int k = 0; k < used; ++k)
    if (cudaStreamWaitEvent(pool->s[k], pool->fork, 0) != cudaSuccess) return fail(WRFGPU_ERR_CUDA, "fork wait failed");
  int first_err = WRFGPU_OK;
  std::string first_msg;
  // members to streams, largest first onto the least loaded stream (cells)
  std::vector<int> order(n), stream_of(n);
  for (int m = 0; m < n; ++m) order[m] = m;
  auto cells = [&](int m) { return (double)params[m].nx * params[m].ny * params[m].nz; };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells(a) > cells(b); });
  std::vector<double> load(used, 0.0);
  for (int m : order) {
    int best = 0;
    for (int k = 1; k < used; ++k)
      if (load[k] < load[best]) best = k;
    stream_of[m] = best;
    load[best] += cells(m);
  }
  for (int m = 0; m < n; ++m) {
    rc = wrfgpu_rk3_step(&params[m], &metrics[m], &in[m], &out[m], lead_seconds[m], workspace[m], workspace_bytes[m],
                         pool->s[stream_of[m]]);
    if (rc && first_err == WRFGPU_OK) {
      first_err = rc;
      first_msg = "member " + std::to_string(m) + ": " + g_last_error;
    }
  }
  // always join, so `stream` never runs ahead of (or leaves dangling) member work
  for (int k = 0; k < used; ++k) {
    if (cudaEventRecord(pool->join[k], pool->s[k]) != cudaSuccess ||
        cudaStreamWaitEvent(stream, pool->join[k], 0) != cudaSuccess)
      return fail(WRFGPU_ERR_CUDA, "join failed");
  }
  if (first_err) return fail(first_err, first_msg);
  g_last_error.clear();
  return WRFGPU_OK;
}

// ---------------------------------------------------------------------------
// Tile-shape tuner: times whole steps for the candidate shapes on this grid.
// ---------------------------------------------------------------------------
extern "C" int wrfgpu_autotune(wrfgpu_step_params *pp, const wrfgpu_metrics *mm, const wrfgpu_step_inputs *in,
                               const wrfgpu_step_outputs *out, void *workspace, size_t workspace_bytes,
                               cudaStream_t stream) {
  if (pp == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "params is NULL");
  int rc = wrfgpu_step_params_validate(pp);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return fail(WRFGPU_ERR_CUDA, "cannot create timing events");
  auto time_steps = [&](const wrfgpu_step_params &p, float *ms) -> int {
    int r = wrfgpu_rk3_step(&p, mm, in, out, NAN, workspace, workspace_bytes, stream);  // warm-up
    if (r) return r;
    cudaEventRecord(e0, stream);
    for (int t = 0; t < 3 && r == WRFGPU_OK; ++t)
      r = wrfgpu_rk3_step(&p, mm, in, out, NAN, workspace, workspace_bytes, stream);
    cudaEventRecord(e1, stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) return fail(WRFGPU_ERR_CUDA, "timing synchronise failed");
    cudaEventElapsedTime(ms, e0, e1);
    return r;
  };
  wrfgpu_step_params best = *pp;
  float best_ms = 1e30f;
  // column block shapes first (march levels at the default), then march levels;
  // width 1 is the one-thread-per-column kernel (its lane count is unused)
  for (int cw : COL_TX_CHOICES) {
    for (int l : COL_TY_CHOICES) {
      if (rc) break;
      if (cw == 1 && l != COL_TY_CHOICES[0]) continue;
      wrfgpu_step_params p = *pp;
      p.column_width = cw;
      p.column_lanes = l;
      p.march_levels = 0;
      float ms = 0.f;
      rc = time_steps(p, &ms);
      if (rc) break;
      if (ms < best_ms) { best_ms = ms; best = p; }
    }
  }
  for (int kcand : MARCH_KC_CHOICES) {
    if (rc) break;
    wrfgpu_step_params p = best;
    p.march_levels = kcand;
    float ms = 0.f;
    rc = time_steps(p, &ms);
    if (rc) break;
    if (ms < best_ms) { best_ms = ms; best = p; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  pp->column_lanes = best.column_lanes;
  pp->column_width = best.column_width;
  pp->march_levels = best.march_levels;
  g_last_error.clear();
  return WRFGPU_OK;
}

// ---------------------------------------------------------------------------
// The scalar advection operator and its adjoint, standalone.
// ---------------------------------------------------------------------------
namespace {
int adv_op_check(const wrfgpu_step_params *p, const wrfgpu_metrics *m, const void *a, const void *ru, const void *rv,
                 const void *rom, const void *b) {
  if (p == nullptr || m == nullptr || a == nullptr || ru == nullptr || rv == nullptr || rom == nullptr || b == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "an argument is NULL");
  if (m->msftx == nullptr || m->rdnw == nullptr || m->fnm == nullptr || m->fnp == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "metrics msftx/rdnw/fnm/fnp are needed");
  return wrfgpu_step_params_validate(p);
}
}  // namespace

// ---------------------------------------------------------------------------
// One acoustic substep on caller-held work state and stage constants, and its
// vector-Jacobian product.
// ---------------------------------------------------------------------------
namespace {

struct AcLayout {
  double *rmsf[6];
  double *dvdxi, *hdiv;
  double *x1[14];  // forward output copy (vjp only), in wrfgpu_acoustic_work order
  AdjScratch s;
};

// element counts of the work arrays in wrfgpu_acoustic_work order
void ac_counts(const Dims &d, size_t n[14]) {
  const size_t c[14] = {d.u, d.v, d.w, d.w, d.m, d.m, d.m, d.m, d.m, d.w, d.s2, d.s2, d.s2, d.s2};
  for (int q = 0; q < 14; ++q) n[q] = c[q];
}

void ac_carve(const wrfgpu_step_params &p, Carver &cv, AcLayout &L) {
  const Dims d = dims_of(p);
  L.rmsf[0] = cv.take(d.s2); L.rmsf[1] = cv.take(d.s2);
  L.rmsf[2] = cv.take(d.su); L.rmsf[3] = cv.take(d.su);
  L.rmsf[4] = cv.take(d.sv); L.rmsf[5] = cv.take(d.sv);
  L.dvdxi = cv.take(d.m); L.hdiv = cv.take(d.m);
  size_t n[14];
  ac_counts(d, n);
  for (int q = 0; q < 14; ++q) L.x1[q] = cv.take(n[q]);
  L.s.gthw = cv.take(d.m); L.s.gtend = cv.take(d.m); L.s.gdv = cv.take(d.m);
  L.s.grhs = cv.take(d.w); L.s.gws = cv.take(d.w); L.s.gww = cv.take(d.w);
  for (int n = 0; n < 3; ++n) {
    L.s.fu[n] = cv.take(d.u);
    L.s.fv[n] = cv.take(d.v);
  }
}

double *const *work_ptrs(const wrfgpu_acoustic_work &x, double *out[14]) {
  double *v[14] = {x.u, x.v, x.w, x.ph, x.theta_w, x.t_2ave, x.p, x.pm1, x.al, x.ww, x.mu, x.muts, x.muave, x.mudf};
  for (int q = 0; q < 14; ++q) out[q] = v[q];
  return out;
}

int ac_check(const wrfgpu_step_params *p, const wrfgpu_metrics *m, const wrfgpu_acoustic_consts *c, size_t ws_bytes,
             const void *ws) {
  if (p == nullptr || m == nullptr || c == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "params/metrics/consts is NULL");
  int rc = wrfgpu_step_params_validate(p);
  if (rc) return rc;
  if (p->run_boundary && (c->u_target == nullptr || c->v_target == nullptr))
    return fail(WRFGPU_ERR_NULL_POINTER, "run_boundary needs the u_target / v_target work targets");
  if (p->w_damping != 0)
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "the standalone acoustic substep has no w_damping CFL term");
  const double *need[] = {c->u_tend, c->v_tend, c->t_tend, c->rw_tend, c->ph_tend, c->alt, c->pb, c->c2a, c->cqu,
                          c->cqv, c->cqw, c->php, c->pt1, c->a, c->alpha, c->gamma, c->ww_1, c->mut, c->muu,
                          c->muv, c->u_1, c->v_1, c->w_save, c->theta, c->phb0};
  for (const double *q : need)
    if (q == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "a stage constant pointer is NULL (only mu_tend may be)");
  size_t need_bytes = 0;
  wrfgpu_acoustic_workspace_size(p, &need_bytes);
  if (ws == nullptr || ws_bytes < need_bytes)
    return fail(WRFGPU_ERR_WORKSPACE, "workspace is NULL or smaller than wrfgpu_acoustic_workspace_size()");
  return WRFGPU_OK;
}

Acoustic ac_state(const wrfgpu_acoustic_consts &c, double *const w[14]) {
  Acoustic A{};
  A.u = w[0]; A.v = w[1]; A.w = w[2]; A.ph = w[3]; A.theta_w = w[4]; A.t2ave = w[5]; A.p = w[6]; A.pm1 = w[7];
  A.al = w[8]; A.ww = w[9]; A.mu = w[10]; A.muts = w[11]; A.muave = w[12]; A.mudf = w[13];
  A.u_tend = c.u_tend; A.v_tend = c.v_tend; A.t_tend = c.t_tend; A.rw_tend = c.rw_tend; A.ph_tend = c.ph_tend;
  A.alt = c.alt; A.pb = c.pb; A.c2a = c.c2a; A.cqu = c.cqu; A.cqv = c.cqv; A.cqw = c.cqw; A.php = c.php;
  A.pt1 = c.pt1; A.a = c.a; A.alpha = c.alpha; A.gamma = c.gamma; A.ww_1 = c.ww_1;
  A.mut = c.mut; A.muu = c.muu; A.muv = c.muv; A.muus = c.muu; A.muvs = c.muv; A.mu_tend = c.mu_tend;
  A.u_1 = c.u_1; A.v_1 = c.v_1; A.w_save = c.w_save; A.theta_s = c.theta; A.phb0 = c.phb0;
  return A;
}

// The boundary relaxation of one substep (as the step sets it up).
BdyArgs ac_bdy(const wrfgpu_step_params &p, const wrfgpu_acoustic_consts &c, double dts) {
  BdyArgs ba{};
  ba.active = p.run_boundary ? 1 : 0;
  if (ba.active) {
    const double strength = (p.normal_bdy_relax_strength < 0.0) ? 20.0 : p.normal_bdy_relax_strength;
    ba.u_target = c.u_target;
    ba.v_target = c.v_target;
    ba.sub_ratio = strength * (p.dt != 0.0 ? dts / p.dt : 0.0);
    ba.spec_zone = 1;
    ba.relax_zone = 4;
    set_bdy_weights(ba);
  }
  return ba;
}

// Launch one forward substep over the work arrays w[14] (in place).
int ac_forward(const wrfgpu_step_params &p, const Grid &g, const wrfgpu_acoustic_consts &c, double *const w[14],
               double dts, const AcLayout &L, cudaStream_t stream) {
  Acoustic A = ac_state(c, w);
  const int specified = (p.run_boundary && !p.bc_ideal) ? 1 : 0;
  BdyArgs ba = ac_bdy(p, c, dts);
  ColArgs ca{};
  ca.dts = dts; ca.epssm = p.epssm; ca.specified = specified; ca.top_lid = p.top_lid; ca.w_damping = 0;
  ca.damp_opt = p.damp_opt; ca.dampcoef = p.dampcoef; ca.zdamp = p.zdamp;
  ca.rzdamp = (p.zdamp != 0.0 && std::isfinite(1.0 / p.zdamp)) ? 1.0 / p.zdamp : 0.0;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  k_advance_uv<false><<<grd(nx + 1, ny + 1, (nz + UV_KC - 1) / UV_KC), blk2(), 0, stream>>>(g, A, dts, p.top_lid, ba);
  if (int rc = check_launch("k_advance_uv")) return rc;
  k_div_h<<<grd(nx, ny, nz), blk2(), 0, stream>>>(g, A, specified, L.dvdxi, L.hdiv);
  if (int rc = check_launch("k_div_h")) return rc;
  const size_t smem = column_tiled_smem_bytes(nz, COL_TX);
  auto kColumn = k_column_tiled<COL_TX, COL_TY>;
  if (cudaFuncSetAttribute(kColumn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return fail(WRFGPU_ERR_CUDA, "cannot reserve shared memory for k_column_tiled (nz too large)");
  kColumn<<<dim3((nx + COL_TX - 1) / COL_TX, ny, 1), dim3(COL_TX, COL_TY, 1), smem, stream>>>(g, A, ca, L.dvdxi,
                                                                                             L.hdiv);
  return check_launch("k_column_tiled");
}

Grid ac_grid(const wrfgpu_step_params &p, const wrfgpu_metrics &m, const AcLayout &L) {
  Grid g = make_grid(p, m, nullptr);
  g.rmsftx = L.rmsf[0]; g.rmsfty = L.rmsf[1]; g.rmsfux = L.rmsf[2]; g.rmsfuy = L.rmsf[3];
  g.rmsfvx = L.rmsf[4]; g.rmsfvy = L.rmsf[5];
  return g;
}

}  // namespace

extern "C" int wrfgpu_acoustic_workspace_size(const wrfgpu_step_params *p, size_t *bytes) {
  if (p == nullptr || bytes == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "params/bytes is NULL");
  int rc = wrfgpu_step_params_validate(p);
  if (rc) return rc;
  Carver cv{nullptr, 0, 0, true};
  AcLayout L;
  ac_carve(*p, cv, L);
  *bytes = cv.off + 256;
  return WRFGPU_OK;
}

extern "C" int wrfgpu_acoustic_substep(const wrfgpu_step_params *p, const wrfgpu_metrics *m,
                                       const wrfgpu_acoustic_consts *c, wrfgpu_acoustic_work *x, double dts,
                                       void *workspace, size_t workspace_bytes, cudaStream_t stream) {
  int rc = ac_check(p, m, c, workspace_bytes, workspace);
  if (rc) return rc;
  if (x == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "work state is NULL");
  double *w[14];
  work_ptrs(*x, w);
  for (double *q : w)
    if (q == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "a work state pointer is NULL");
  Carver cv{reinterpret_cast<char *>(workspace), 0, workspace_bytes, false};
  AcLayout L;
  ac_carve(*p, cv, L);
  Grid g = ac_grid(*p, *m, L);
  k_recip_msf<<<grd(p->nx + 1, p->ny + 1, 1), blk2(), 0, stream>>>(g, L.rmsf[0], L.rmsf[1], L.rmsf[2], L.rmsf[3],
                                                                 L.rmsf[4], L.rmsf[5]);
  if ((rc = check_launch("k_recip_msf"))) return rc;
  if ((rc = ac_forward(*p, g, *c, w, dts, L, stream))) return rc;
  g_last_error.clear();
  return WRFGPU_OK;
}

extern "C" int wrfgpu_acoustic_substep_vjp(const wrfgpu_step_params *p, const wrfgpu_metrics *m,
                                           const wrfgpu_acoustic_consts *c, const wrfgpu_acoustic_work *x,
                                           const wrfgpu_acoustic_work *x_out, const wrfgpu_acoustic_work *cot_out,
                                           wrfgpu_acoustic_work *cot_in, wrfgpu_acoustic_tend_cot *cot_tend,
                                           double dts, void *workspace, size_t workspace_bytes,
                                           cudaStream_t stream) {
  int rc = ac_check(p, m, c, workspace_bytes, workspace);
  if (rc) return rc;
  if (x == nullptr || cot_out == nullptr || cot_in == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "work state or cotangent is NULL");
  double *xin[14], *co[14], *ci[14];
  work_ptrs(*x, xin);
  work_ptrs(*cot_out, co);
  work_ptrs(*cot_in, ci);
  for (int q = 0; q < 14; ++q)
    if (xin[q] == nullptr || co[q] == nullptr || ci[q] == nullptr)
      return fail(WRFGPU_ERR_NULL_POINTER, "a work state or cotangent pointer is NULL");
  const Dims d = dims_of(*p);
  Carver cv{reinterpret_cast<char *>(workspace), 0, workspace_bytes, false};
  AcLayout L;
  ac_carve(*p, cv, L);
  Grid g = ac_grid(*p, *m, L);
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  k_recip_msf<<<grd(nx + 1, ny + 1, 1), blk2(), 0, stream>>>(g, L.rmsf[0], L.rmsf[1], L.rmsf[2], L.rmsf[3],
                                                           L.rmsf[4], L.rmsf[5]);
  if ((rc = check_launch("k_recip_msf"))) return rc;
  // forward output X' = F(X): the caller's, or recomputed into the workspace
  size_t n[14];
  ac_counts(d, n);
  double *x1[14];
  if (x_out != nullptr) {
    work_ptrs(*x_out, x1);
    for (double *q : x1)
      if (q == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "an x_out pointer is NULL");
  } else {
    for (int q = 0; q < 14; ++q) {
      x1[q] = L.x1[q];
      if (cudaMemcpyAsync(L.x1[q], xin[q], n[q] * sizeof(double), cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
        return fail(WRFGPU_ERR_CUDA, "work state copy failed");
    }
    if ((rc = ac_forward(*p, g, *c, L.x1, dts, L, stream))) return rc;
  }
  const int specified = (p->run_boundary && !p->bc_ideal) ? 1 : 0;
  if (specified && x_out != nullptr) {  // the forward dvdxi (the drain limiter's input) from the stored output
    Acoustic A = ac_state(*c, x1);
    k_div_h<<<grd(nx, ny, nz), blk2(), 0, stream>>>(g, A, 1, L.dvdxi, L.hdiv);
    if ((rc = check_launch("k_div_h"))) return rc;
  }
  // the cotangents the advance_uv transpose accumulates into start from zero
  for (int q : {6, 8, 13})
    if (cudaMemsetAsync(ci[q], 0, n[q] * sizeof(double), stream) != cudaSuccess)
      return fail(WRFGPU_ERR_CUDA, "cotangent clear failed");
  AdjColArgs a{};
  if (cot_tend != nullptr)
    a.tc = AdjTend{cot_tend->u_tend, cot_tend->v_tend, cot_tend->t_tend, cot_tend->rw_tend, cot_tend->ph_tend,
                   cot_tend->mu_tend};
  a.x0_muts = xin[11];
  a.dvdxi = L.dvdxi;
  a.mu_tend = c->mu_tend;
  a.specified = specified;
  a.x1 = AcWorkR{x1[0], x1[1], x1[2], x1[3], x1[4], x1[5], x1[6], x1[7], x1[8], x1[9], x1[10], x1[11], x1[12], x1[13]};
  a.co = AcWorkR{co[0], co[1], co[2], co[3], co[4], co[5], co[6], co[7], co[8], co[9], co[10], co[11], co[12], co[13]};
  a.ci = AcWork{ci[0], ci[1], ci[2], ci[3], ci[4], ci[5], ci[6], ci[7], ci[8], ci[9], ci[10], ci[11], ci[12], ci[13]};
  a.s = L.s;
  a.alt = c->alt; a.c2a = c->c2a; a.cqw = c->cqw; a.theta_s = c->theta; a.pt1 = c->pt1;
  a.a = c->a; a.alpha = c->alpha; a.gamma = c->gamma; a.mut = c->mut;
  a.col.dts = dts; a.col.epssm = p->epssm; a.col.top_lid = p->top_lid; a.col.damp_opt = p->damp_opt;
  a.col.dampcoef = p->dampcoef; a.col.zdamp = p->zdamp;
  a.col.rzdamp = (p->zdamp != 0.0 && std::isfinite(1.0 / p->zdamp)) ? 1.0 / p->zdamp : 0.0;
  k_adj_column<<<grd(nx, ny, 1), blk2(), 0, stream>>>(g, a);
  if ((rc = check_launch("k_adj_column"))) return rc;
  AdjFaceArgs fa{L.s.gtend, L.s.gdv, c->theta, co[0], co[1], ci[0], ci[1], ac_bdy(*p, *c, dts)};
  k_adj_faces<<<grd(nx + 1, ny + 1, nz), blk2(), 0, stream>>>(g, fa);
  if ((rc = check_launch("k_adj_faces"))) return rc;
  AdjUVArgs ua{};
  ua.gu_tend = cot_tend != nullptr ? cot_tend->u_tend : nullptr;
  ua.gv_tend = cot_tend != nullptr ? cot_tend->v_tend : nullptr;
  ua.gu = ci[0]; ua.gv = ci[1];
  ua.alt = c->alt; ua.pb = c->pb; ua.php = c->php; ua.cqu = c->cqu; ua.cqv = c->cqv; ua.muu = c->muu; ua.muv = c->muv;
  ua.ci_p = ci[6]; ua.ci_ph = ci[3]; ua.ci_al = ci[8]; ua.ci_muts = ci[11]; ua.ci_mudf = ci[13];
  for (int n = 0; n < 3; ++n) {
    ua.fu[n] = L.s.fu[n];
    ua.fv[n] = L.s.fv[n];
  }
  ua.dts = dts;
  ua.top_lid = p->top_lid;
  k_adj_uv_faces<<<grd(nx + 1, ny + 1, nz), blk2(), 0, stream>>>(g, ua);
  if ((rc = check_launch("k_adj_uv_faces"))) return rc;
  k_adj_uv_cells<<<grd(nx, ny, nz + 1), blk2(), 0, stream>>>(g, ua);
  if ((rc = check_launch("k_adj_uv_cells"))) return rc;
  k_adj_uv_cols<<<grd(nx, ny, 1), blk2(), 0, stream>>>(g, ua);
  if ((rc = check_launch("k_adj_uv_cols"))) return rc;
  g_last_error.clear();
  return WRFGPU_OK;
}

// ---------------------------------------------------------------------------
// The end-of-step lateral boundary pass.
// ---------------------------------------------------------------------------
namespace {

// The state and strip checks shared by the boundary pass and the epilogue.
int epilogue_check(const wrfgpu_step_params *p, const wrfgpu_step_inputs *in, const wrfgpu_lbc_leaves *lv,
                   const wrfgpu_step_outputs *out, bool boundary, bool spec_only, double lead_seconds) {
  int rc = wrfgpu_step_params_validate(p);
  if (rc) return rc;
  if (boundary && (p->spec_zone != 1 || p->relax_zone != 4))
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "boundary zones other than spec_zone=1, relax_zone=4 are not built");
  if (boundary && !std::isfinite(lead_seconds))
    return fail(WRFGPU_ERR_UNSUPPORTED_CONFIG, "lead_seconds must be finite");
  const double *req_in[] = {in->u, in->v, in->w, in->theta, in->p_total, in->p_perturbation, in->ph_total,
                            in->ph_perturbation, in->mu_total, in->mu_perturbation};
  double *req_out[] = {out->u, out->v, out->w, out->theta, out->p_total, out->p_perturbation, out->ph_total,
                       out->ph_perturbation, out->mu_total, out->mu_perturbation};
  for (int k = 0; k < 10; ++k) {
    if (req_in[k] == nullptr || req_out[k] == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "a state pointer is NULL");
    if ((const double *)req_out[k] == req_in[k]) return fail(WRFGPU_ERR_BAD_SHAPE, "out must not alias the input state");
  }
  for (int s = 0; s < 6; ++s)
    if ((in->q[s] == nullptr) != (out->q[s] == nullptr))
      return fail(WRFGPU_ERR_NULL_POINTER, "a moisture species needs both its input and its output");
  if (!boundary) return WRFGPU_OK;
  if (lv == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "the boundary pass needs the strips");
  const double *need[] = {lv->u, lv->v, lv->theta, lv->mu, lv->mub, lv->ph, lv->phb};
  for (const double *q : need)
    if (q == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "the u, v, theta, mu, mub, ph and phb strips are needed");
  if (!spec_only && (lv->w == nullptr || lv->p == nullptr || lv->pb == nullptr))
    return fail(WRFGPU_ERR_NULL_POINTER, "the full pass needs the w, p and pb strips");
  if (lv->ntime < 1 || lv->width < 1 || lv->side_len < (p->nx > p->ny ? p->nx + 1 : p->ny + 1))
    return fail(WRFGPU_ERR_BAD_SHAPE, "strips must be (ntime >= 1, 4, width >= 1, levels, side_len >= max(nx, ny) + 1)");
  for (int s = 0; s < 6; ++s)
    if (lv->q[s] != nullptr && in->q[s] == nullptr)
      return fail(WRFGPU_ERR_NULL_POINTER, "a forced moisture species needs its input and output");
  return WRFGPU_OK;
}

// One launch per field (or a copy where nothing touches it): the boundary
// pass (when `boundary`) with the guards fused before and after it (when
// `guards`; `gs` / `after` are the theta limiter's scalars and partials).
int epilogue_fields(const wrfgpu_step_params *p, const wrfgpu_step_inputs *org, const wrfgpu_step_inputs *in,
                    const wrfgpu_lbc_leaves *lv, const wrfgpu_step_outputs *out, double lead_seconds,
                    const double *lead_dev, bool guards, bool boundary, bool spec_only, const GuardScalars *gs,
                    double *after, int *theta_slots, cudaStream_t stream) {
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  BdyLeaf nolf{};
  auto leaf = [&](const double *x) -> BdyLeaf {
    if (!boundary || x == nullptr) return nolf;
    // strips at the lead (boundary_apply.py:329-345), on the host or read
    // from the device lead by the kernels
    BdyLeaf b{x, lv->ntime, lv->width, lv->side_len, 0, 0, 0.0, lead_dev, 0.0, p->update_cadence_s};
    if (lead_dev == nullptr) leaf_time_weights(lead_seconds, p->update_cadence_s, lv->ntime, b.lo, b.hi, b.alpha);
    return b;
  };
  // dt*fcx, dt*gcx of the relax rows (boundary_apply.py:666-688, spec_exp 0)
  LbcJob base{};
  for (int b = 1; b <= 3; ++b) {
    const double dt = p->dt;
    const double linear = (double)(p->spec_zone + p->relax_zone - (b + 1)) / (double)(p->relax_zone - 1);
    const double fcx = 0.1 / dt * (linear > 0.0 ? linear : 0.0) * 1.0;
    const double gcx = 1.0 / dt / 50.0 * (linear > 0.0 ? linear : 0.0) * 1.0;
    base.wf[b] = dt * fcx;
    base.wg[b] = dt * gcx;
  }
  const int ring = boundary ? (spec_only ? 1 : 2) : 0;
  // the field jobs, launched together at the end: the elementwise parts, then the ring bands
  LbcBatch inner{}, rings{};
  // shared x / y grids: the widest field (nx + 1 by ny + 1); the ring band of the largest field
  const dim3 inner_grid = grd(nx + 1, ny + 1, 1);
  const bool small = nx + 1 < 8 || ny + 1 < 8;
  const int ring_gx = (ring_cells(nx + 1, ny + 1, small ? 1 : 0) + LBC_RING_THREADS - 1) / LBC_RING_THREADS;
  const int post_fin = (guards && boundary) ? GUARD_FINITE : GUARD_NONE;
  auto copy = [&](double *o, const double *x, size_t n) -> int {
    if (o == x) return WRFGPU_OK;
    if (cudaMemcpyAsync(o, x, n * sizeof(double), cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      return fail(WRFGPU_ERR_CUDA, "epilogue copy failed");
    return WRFGPU_OK;
  };
  // one field: x (x2: a pair's perturbation) into o (o2), levels zl, extent yl x xl
  auto run = [&](const double *x, const double *x2, double *o, double *o2, const double *o_org, const double *o_org2,
                 const double *l1, const double *l2, int zl, int yl, int xl, int rg, int pre, int post,
                 int clamp) -> int {
    const size_t n = (size_t)zl * yl * xl;
    if (rg == 0 && pre == GUARD_NONE && post == GUARD_NONE) {
      int rc = copy(o, x, n);
      if (!rc && x2 != nullptr) rc = copy(o2, x2, n);
      return rc;
    }
    LbcJob a = base;
    a.x = x; a.x2 = x2; a.out = o; a.out2 = o2;
    a.leaf = leaf(l1);
    a.leaf2 = leaf(l2 != nullptr ? l2 : l1);
    a.zl = zl; a.yl = yl; a.xl = xl;
    a.ring = rg; a.clamp = clamp;
    a.pre = pre; a.post = post;
    a.org = o_org; a.org2 = o_org2;
    a.mu_next = in->mu_total;
    a.gs = gs;
    a.after = after;
    a.all_ring = (rg && (xl < 8 || yl < 8)) ? 1 : 0;
    int inner_blocks = 0;
    if (!a.all_ring) {
      const int q = inner.njobs++;
      inner.job[q] = a;
      inner.slot0[q] = 0;
      inner_blocks = (int)(inner_grid.x * inner_grid.y);
    }
    int ring_blocks = 0;
    if (rg) {
      if (ring_cells(xl, yl, a.all_ring) > ring_gx * LBC_RING_THREADS)
        return fail(WRFGPU_ERR_BAD_SHAPE, "a field's ring band exceeds the shared ring grid");
      const int q = rings.njobs++;
      rings.job[q] = a;
      rings.slot0[q] = inner_blocks;
      rings.start[q + 1] = rings.start[q] + zl;
      ring_blocks = ring_gx * zl;
    }
    if (pre == GUARD_THETA) *theta_slots = inner_blocks + ring_blocks;
    return WRFGPU_OK;
  };
  const bool geo = p->force_geopotential != 0;
  const wrfgpu_step_inputs *O = org;
  const double *nul = nullptr;
  int rc;
  if ((rc = run(in->u, nul, out->u, nullptr, O ? O->u : nul, nul, lv ? lv->u : nul, nul, nz, ny, nx + 1, ring,
                GUARD_NONE, post_fin, 0)))
    return rc;
  if ((rc = run(in->v, nul, out->v, nullptr, O ? O->v : nul, nul, lv ? lv->v : nul, nul, nz, ny + 1, nx, ring,
                GUARD_NONE, post_fin, 0)))
    return rc;
  // WRF's specified cadence leaves w and p to the step (boundary_apply.py:217-220, 290)
  const int ring_wp = spec_only ? 0 : ring;
  if ((rc = run(in->w, nul, out->w, nullptr, O ? O->w : nul, nul, lv ? lv->w : nul, nul, nz + 1, ny, nx, ring_wp,
                GUARD_NONE, post_fin, 0)))
    return rc;
  if ((rc = run(in->theta, nul, out->theta, nullptr, O ? O->theta : nul, nul, lv ? lv->theta : nul, nul, nz, ny, nx,
                ring, guards ? GUARD_THETA : GUARD_NONE, post_fin, 0)))
    return rc;
  if ((rc = run(in->p_total, in->p_perturbation, out->p_total, out->p_perturbation, O ? O->p_total : nul,
                O ? O->p_perturbation : nul, lv ? lv->p : nul, lv ? lv->pb : nul, nz, ny, nx, ring_wp, GUARD_NONE,
                post_fin, 0)))
    return rc;
  if ((rc = run(in->mu_total, in->mu_perturbation, out->mu_total, out->mu_perturbation, O ? O->mu_total : nul,
                O ? O->mu_perturbation : nul, lv ? lv->mu : nul, lv ? lv->mub : nul, 1, ny, nx, ring,
                guards ? GUARD_MASS : GUARD_NONE, (guards && boundary) ? GUARD_MASS : GUARD_NONE, 0)))
    return rc;
  // the nested child's geopotential is left to the dynamics (boundary_apply.py:270-307)
  const int ring_ph = (geo || spec_only) ? ring : 0;
  if ((rc = run(in->ph_total, in->ph_perturbation, out->ph_total, out->ph_perturbation, O ? O->ph_total : nul,
                O ? O->ph_perturbation : nul, lv ? lv->ph : nul, lv ? lv->phb : nul, nz + 1, ny, nx, ring_ph,
                GUARD_NONE, post_fin, 0)))
    return rc;
  for (int s = 0; s < 6; ++s) {
    if (in->q[s] == nullptr) continue;
    const bool forced = boundary && lv->q[s] != nullptr;
    const int post = (s == 0 && guards && boundary) ? GUARD_RATIO : GUARD_NONE;
    if ((rc = run(in->q[s], nul, out->q[s], nullptr, O ? O->q[s] : nul, nul, forced ? lv->q[s] : nul, nul, nz, ny, nx,
                  forced ? 2 : 0, guards ? GUARD_RATIO : GUARD_NONE, post, forced ? 1 : 0)))
      return rc;
  }
  if (inner.njobs > 0) {
    k_lbc_fields<<<dim3(inner_grid.x, inner_grid.y, inner.njobs), blk2(), 0, stream>>>(inner);
    if ((rc = check_launch("k_lbc_fields"))) return rc;
  }
  if (rings.njobs > 0) {
    k_lbc_rings<<<dim3(ring_gx, rings.start[rings.njobs], 1), dim3(LBC_RING_THREADS, 1, 1), 0, stream>>>(rings);
    if ((rc = check_launch("k_lbc_rings"))) return rc;
  }
  return WRFGPU_OK;
}

// Workspace layout of wrfgpu_step_epilogue.
struct EpilogueWs {
  size_t scalars, partials, after, total;
  int nparts, nafter;
};

EpilogueWs epilogue_ws(const wrfgpu_step_params &p) {
  EpilogueWs w{};
  const long long n = (long long)p.nz * p.ny * p.nx;
  const long long want = (n + GUARD_THREADS - 1) / GUARD_THREADS;
  w.nparts = (int)(want < 148 * 8 ? (want < 1 ? 1 : want) : 148 * 8);
  // the theta job's blocks: the elementwise kernel's and the ring band's (at most)
  const dim3 g = grd(p.nx + 1, p.ny + 1, 1);
  const int rb = (ring_cells(p.nx + 1, p.ny + 1, 1) + LBC_RING_THREADS - 1) / LBC_RING_THREADS;
  w.nafter = (int)(g.x * g.y * g.z) + rb * p.nz;
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  w.scalars = 0;
  w.partials = up(sizeof(GuardScalars));
  w.after = w.partials + up((size_t)w.nparts * sizeof(GuardPartial));
  w.total = w.after + up((size_t)w.nafter * sizeof(double));
  return w;
}

}  // namespace

extern "C" int wrfgpu_apply_lateral_boundaries(const wrfgpu_step_params *p, const wrfgpu_step_inputs *in,
                                               const wrfgpu_lbc_leaves *lv, const wrfgpu_step_outputs *out,
                                               double lead_seconds, int dry_spec_only, cudaStream_t stream) {
  if (p == nullptr || in == nullptr || lv == nullptr || out == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "params/inputs/leaves/outputs is NULL");
  int rc = epilogue_check(p, in, lv, out, true, dry_spec_only != 0, lead_seconds);
  if (rc) return rc;
  int slots = 0;
  rc = epilogue_fields(p, nullptr, in, lv, out, lead_seconds, nullptr, false, true, dry_spec_only != 0, nullptr,
                       nullptr, &slots, stream);
  if (rc) return rc;
  g_last_error.clear();
  return WRFGPU_OK;
}

extern "C" int wrfgpu_step_epilogue_workspace_size(const wrfgpu_step_params *p, size_t *bytes) {
  if (p == nullptr || bytes == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "params/bytes is NULL");
  int rc = wrfgpu_step_params_validate(p);
  if (rc) return rc;
  *bytes = epilogue_ws(*p).total;
  g_last_error.clear();
  return WRFGPU_OK;
}

namespace {

// The step epilogue at a host lead, or (lead_dev set) at a device-resident
// lead that the boundary kernels read.
int step_epilogue_impl(const wrfgpu_step_params *p, const wrfgpu_step_inputs *origin, const wrfgpu_step_inputs *next,
                       const wrfgpu_lbc_leaves *lv, const wrfgpu_step_outputs *out, double lead_seconds,
                       const double *lead_dev, int disable_guards, wrfgpu_theta_limiter_diag *diag, void *ws,
                       size_t ws_bytes, cudaStream_t stream) {
  if (p == nullptr || next == nullptr || out == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "params/next/out is NULL");
  const bool guards = disable_guards == 0;
  const bool boundary = p->run_boundary != 0;
  // _specified_bdy_cadence_active (operational_mode.py:2478-2491)
  const bool spec_only = boundary && !p->bc_ideal && p->force_geopotential && p->specified_bdy_cadence;
  int rc = epilogue_check(p, next, lv, out, boundary, spec_only, lead_seconds);
  if (rc) return rc;
  if (guards) {
    if (origin == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "the guards need the origin state");
    const double *req[] = {origin->u, origin->v, origin->w, origin->theta, origin->p_total, origin->p_perturbation,
                           origin->ph_total, origin->ph_perturbation, origin->mu_total, origin->mu_perturbation};
    for (const double *q : req)
      if (q == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "an origin state pointer is NULL");
    for (int s = 0; s < 6; ++s)
      if (next->q[s] != nullptr && origin->q[s] == nullptr)
        return fail(WRFGPU_ERR_NULL_POINTER, "a guarded moisture species needs its origin");
  }
  const EpilogueWs w = epilogue_ws(*p);
  if (guards && (ws == nullptr || ws_bytes < w.total || ((uintptr_t)ws & 255) != 0))
    return fail(WRFGPU_ERR_WORKSPACE, "workspace is NULL, too small or not 256-byte aligned");
  GuardScalars *gs = nullptr;
  double *after = nullptr;
  if (guards) {
    char *base = (char *)ws;
    gs = (GuardScalars *)(base + w.scalars);
    GuardPartial *part = (GuardPartial *)(base + w.partials);
    after = (double *)(base + w.after);
    k_guard_reduce<<<w.nparts, GUARD_THREADS, 0, stream>>>(next->theta, origin->theta, next->mu_total, p->nz, p->ny,
                                                           p->nx, part);
    if ((rc = check_launch("k_guard_reduce"))) return rc;
    k_guard_finalize<<<1, GUARD_THREADS, 0, stream>>>(part, w.nparts, gs);
    if ((rc = check_launch("k_guard_finalize"))) return rc;
  }
  int slots = 0;
  rc = epilogue_fields(p, guards ? origin : nullptr, next, lv, out, lead_seconds, lead_dev, guards, boundary,
                       spec_only, gs, after, &slots, stream);
  if (rc) return rc;
  if (diag != nullptr) {
    if (guards)
      k_guard_diag<<<1, GUARD_THREADS, 0, stream>>>(after, slots, gs, p->ny, p->nx, diag);
    else
      k_guard_diag_empty<<<1, 1, 0, stream>>>(diag);
    if ((rc = check_launch("k_guard_diag"))) return rc;
  }
  g_last_error.clear();
  return WRFGPU_OK;
}

}  // namespace

extern "C" int wrfgpu_step_epilogue(const wrfgpu_step_params *p, const wrfgpu_step_inputs *origin,
                                    const wrfgpu_step_inputs *next, const wrfgpu_lbc_leaves *lv,
                                    const wrfgpu_step_outputs *out, double lead_seconds, int disable_guards,
                                    wrfgpu_theta_limiter_diag *diag, void *ws, size_t ws_bytes, cudaStream_t stream) {
  return step_epilogue_impl(p, origin, next, lv, out, lead_seconds, nullptr, disable_guards, diag, ws, ws_bytes,
                            stream);
}

extern "C" int wrfgpu_step_epilogue_device_lead(const wrfgpu_step_params *p, const wrfgpu_step_inputs *origin,
                                                const wrfgpu_step_inputs *next, const wrfgpu_lbc_leaves *lv,
                                                const wrfgpu_step_outputs *out, const double *lead_seconds_dev,
                                                int disable_guards, wrfgpu_theta_limiter_diag *diag, void *ws,
                                                size_t ws_bytes, cudaStream_t stream) {
  if (lead_seconds_dev == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "lead_seconds_dev is NULL");
  return step_epilogue_impl(p, origin, next, lv, out, 0.0, lead_seconds_dev, disable_guards, diag, ws, ws_bytes,
                            stream);
}

extern "C" int wrfgpu_flux_advection(const wrfgpu_step_params *p, const wrfgpu_metrics *m, const double *q,
                                     const double *ru, const double *rv, const double *rom, const double *hfac,
                                     const double *vfac, double *tend, cudaStream_t stream) {
  // rom NULL: the horizontal flux divergence alone
  int rc = adv_op_check(p, m, q, ru, rv, rom != nullptr ? rom : ru, tend);
  if (rc) return rc;
  Grid g = make_grid(*p, *m, nullptr);
  AdvOpArgs a{ru, rv, rom, hfac != nullptr ? hfac : m->msftx, vfac};
  k_scalar_adv_op<<<grd(p->nx, p->ny, p->nz), blk2(), 0, stream>>>(g, a, q, tend);
  if (cudaGetLastError() != cudaSuccess) return fail(WRFGPU_ERR_CUDA, "k_scalar_adv_op launch failed");
  g_last_error.clear();
  return WRFGPU_OK;
}

extern "C" int wrfgpu_flux_advection_vjp(const wrfgpu_step_params *p, const wrfgpu_metrics *m, const double *q,
                                         const double *tend_bar, const double *ru, const double *rv,
                                         const double *rom, const double *hfac, const double *vfac, double *q_bar,
                                         double *ru_bar, double *rv_bar, double *rom_bar, cudaStream_t stream) {
  const bool vel = ru_bar != nullptr || rv_bar != nullptr || rom_bar != nullptr;
  // q is read only for the velocities' cotangents; rom NULL: horizontal only
  int rc = adv_op_check(p, m, vel ? q : tend_bar, ru, rv, rom != nullptr ? rom : ru, tend_bar);
  if (rc) return rc;
  if (rom == nullptr && rom_bar != nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "rom_bar needs rom");
  if (q_bar == nullptr && !vel) return fail(WRFGPU_ERR_NULL_POINTER, "q_bar, ru_bar, rv_bar and rom_bar are all NULL");
  Grid g = make_grid(*p, *m, nullptr);
  AdvOpArgs a{ru, rv, rom, hfac != nullptr ? hfac : m->msftx, vfac};
  const int nzl = p->nz + (rom_bar != nullptr ? 1 : 0);
  k_scalar_adv_vjp<<<tgrd(p->nx, p->ny, nzl), tblk(), 0, stream>>>(g, a, vel ? q : tend_bar, tend_bar, q_bar, ru_bar,
                                                                     rv_bar, rom_bar);
  if (cudaGetLastError() != cudaSuccess) return fail(WRFGPU_ERR_CUDA, "k_scalar_adv_vjp launch failed");
  g_last_error.clear();
  return WRFGPU_OK;
}

extern "C" int wrfgpu_w_vertical_advection(const wrfgpu_step_params *p, const wrfgpu_metrics *m, const double *w,
                                           const double *rom, double *tend, cudaStream_t stream) {
  if (p == nullptr || m == nullptr || w == nullptr || rom == nullptr || tend == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "an argument is NULL");
  if (m->rdn == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "metrics rdn is needed");
  int rc = wrfgpu_step_params_validate(p);
  if (rc) return rc;
  Grid g = make_grid(*p, *m, nullptr);
  k_vdiv_w<<<grd(p->nx, p->ny, p->nz + 1), blk2(), 0, stream>>>(g, WColumn{w, rom, p->top_lid}, tend);
  if (cudaGetLastError() != cudaSuccess) return fail(WRFGPU_ERR_CUDA, "k_vdiv_w launch failed");
  g_last_error.clear();
  return WRFGPU_OK;
}

extern "C" int wrfgpu_w_vertical_advection_vjp(const wrfgpu_step_params *p, const wrfgpu_metrics *m,
                                               const double *w, const double *rom, const double *tend_bar,
                                               double *w_bar, double *rom_bar, cudaStream_t stream) {
  if (p == nullptr || m == nullptr || w == nullptr || rom == nullptr || tend_bar == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "an argument is NULL");
  if (w_bar == nullptr && rom_bar == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "w_bar and rom_bar are NULL");
  if (m->rdn == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "metrics rdn is needed");
  int rc = wrfgpu_step_params_validate(p);
  if (rc) return rc;
  Grid g = make_grid(*p, *m, nullptr);
  k_vdiv_w_vjp<<<grd(p->nx, p->ny, p->nz + 1), blk2(), 0, stream>>>(g, WColumn{w, rom, p->top_lid}, tend_bar, w_bar,
                                                                   rom_bar);
  if (cudaGetLastError() != cudaSuccess) return fail(WRFGPU_ERR_CUDA, "k_vdiv_w_vjp launch failed");
  g_last_error.clear();
  return WRFGPU_OK;
}

extern "C" int wrfgpu_scalar_advection(const wrfgpu_step_params *p, const wrfgpu_metrics *m, const double *q,
                                       const double *ru, const double *rv, const double *rom, double *tend,
                                       cudaStream_t stream) {
  return wrfgpu_flux_advection(p, m, q, ru, rv, rom, nullptr, nullptr, tend, stream);
}

extern "C" int wrfgpu_scalar_advection_adjoint(const wrfgpu_step_params *p, const wrfgpu_metrics *m,
                                               const double *tend_bar, const double *ru, const double *rv,
                                               const double *rom, double *q_bar, cudaStream_t stream) {
  return wrfgpu_flux_advection_vjp(p, m, nullptr, tend_bar, ru, rv, rom, nullptr, nullptr, q_bar, nullptr, nullptr,
                                   nullptr, stream);
}

extern "C" int wrfgpu_scalar_advection_vjp(const wrfgpu_step_params *p, const wrfgpu_metrics *m, const double *q,
                                           const double *tend_bar, const double *ru, const double *rv,
                                           const double *rom, double *q_bar, double *ru_bar, double *rv_bar,
                                           double *rom_bar, cudaStream_t stream) {
  return wrfgpu_flux_advection_vjp(p, m, q, tend_bar, ru, rv, rom, nullptr, nullptr, q_bar, ru_bar, rv_bar, rom_bar,
                                   stream);
}

// ---------------------------------------------------------------------------
// Nest coupling: parent -> child interpolation and boundary leaves, child ->
// parent feedback (nesting.cuh).
// ---------------------------------------------------------------------------
namespace {

int nest_interp_check(const wrfgpu_nest_interp *w) {
  if (w == nullptr || w->y0 == nullptr || w->y1 == nullptr || w->x0 == nullptr || w->x1 == nullptr ||
      w->wy == nullptr || w->wx == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "interpolation weights are NULL");
  if (w->child_ny < 1 || w->child_nx < 1 || w->parent_ny < 1 || w->parent_nx < 1)
    return fail(WRFGPU_ERR_BAD_SHAPE, "interpolation extents must be >= 1");
  return WRFGPU_OK;
}

NestInterp nest_interp_of(const wrfgpu_nest_interp *w) {
  return NestInterp{w->y0, w->y1, w->x0, w->x1, w->wy, w->wx, w->child_ny, w->child_nx, w->parent_ny, w->parent_nx};
}

}  // namespace

extern "C" int wrfgpu_nest_interp_field(const wrfgpu_nest_interp *w, const double *parent, int nz, double *child_out,
                                        cudaStream_t stream) {
  int rc = nest_interp_check(w);
  if (rc) return rc;
  if (parent == nullptr || child_out == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "parent/child_out is NULL");
  if (nz < 1 || nz > 65535) return fail(WRFGPU_ERR_BAD_SHAPE, "nz must be in 1..65535");
  const NestInterp ni = nest_interp_of(w);
  k_nest_interp<<<dim3((ni.cnx + 31) / 32, (ni.cny + 3) / 4, nz), dim3(32, 4, 1), 0, stream>>>(ni, parent, child_out);
  if ((rc = check_launch("k_nest_interp"))) return rc;
  g_last_error.clear();
  return WRFGPU_OK;
}

extern "C" int wrfgpu_nest_ring_leaf(const wrfgpu_nest_interp *w, const double *parent, const double *child,
                                     const double *child_sub, int nz, int child_ny, int child_nx, int width,
                                     int side_len, int leaf_z, int leaf_side, double *leaf, cudaStream_t stream) {
  if (child == nullptr || leaf == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "child/leaf is NULL");
  if (w != nullptr) {
    int rc = nest_interp_check(w);
    if (rc) return rc;
    if (parent == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "parent is NULL");
    if (w->child_ny != child_ny || w->child_nx != child_nx)
      return fail(WRFGPU_ERR_BAD_SHAPE, "the weights' child extent differs from the child field's");
  }
  if (nz < 1 || child_ny < 1 || child_nx < 1 || width < 1 || side_len < 1 || leaf_z < 1 || leaf_side < 1 ||
      4 * width > 65535 || 2 * leaf_z > 65535)
    return fail(WRFGPU_ERR_BAD_SHAPE, "bad ring-leaf extents");
  NestRingJob a{};
  if (w != nullptr) a.w = nest_interp_of(w);
  a.w.cny = child_ny;
  a.w.cnx = child_nx;
  a.interp = w != nullptr ? 1 : 0;
  a.parent = parent;
  a.child = child;
  a.child_sub = child_sub;
  a.nzf = nz;
  a.width = width;
  a.side_len = side_len;
  a.lz = leaf_z;
  a.lside = leaf_side;
  a.leaf = leaf;
  k_nest_ring_leaf<<<dim3((leaf_side + 127) / 128, 4 * width, 2 * leaf_z), 128, 0, stream>>>(a);
  int rc = check_launch("k_nest_ring_leaf");
  if (rc) return rc;
  g_last_error.clear();
  return WRFGPU_OK;
}

extern "C" int wrfgpu_nest_feedback(const wrfgpu_nest_feedback_plan *plan, const double *parent, const double *child,
                                    int nz, double *out, double *scratch, cudaStream_t stream) {
  if (plan == nullptr || parent == nullptr || child == nullptr || out == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "plan/parent/child/out is NULL");
  if (plan->npts > 0 && (plan->parent_lin == nullptr || plan->child_lin == nullptr))
    return fail(WRFGPU_ERR_NULL_POINTER, "the plan's index arrays are NULL");
  if (nz < 1 || nz > 65535 || plan->npts < 0 || plan->stencil < 1 || plan->pwe < 1 || plan->psn < 1 ||
      plan->cwe < 1 || plan->csn < 1)
    return fail(WRFGPU_ERR_BAD_SHAPE, "bad feedback extents");
  const bool smooth = plan->smooth != 0 && plan->i_hi > plan->i_lo && plan->j_hi > plan->j_lo;
  if (smooth && scratch == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "the smoother needs a scratch field");
  if (smooth && (plan->i_lo < 1 || plan->j_lo < 1 || plan->i_hi > plan->pwe - 1 || plan->j_hi > plan->psn - 1))
    return fail(WRFGPU_ERR_BAD_SHAPE, "the smoother interior needs a one-cell halo inside the parent field");
  const size_t n = (size_t)nz * plan->psn * plan->pwe;
  if (out != parent && cudaMemcpyAsync(out, parent, n * sizeof(double), cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
    return fail(WRFGPU_ERR_CUDA, "feedback copy failed");
  int rc;
  if (plan->npts > 0) {
    NestFeedback f{plan->parent_lin, plan->child_lin, plan->npts, plan->stencil, plan->pwe, plan->psn, plan->cwe,
                   plan->csn};
    k_nest_feedback<<<dim3((plan->npts + 127) / 128, nz, 1), 128, 0, stream>>>(f, child, out);
    if ((rc = check_launch("k_nest_feedback"))) return rc;
  }
  if (smooth) {
    if (cudaMemcpyAsync(scratch, out, n * sizeof(double), cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      return fail(WRFGPU_ERR_CUDA, "smoother copy failed");
    const dim3 grid((plan->i_hi - plan->i_lo + 31) / 32, (plan->j_hi - plan->j_lo + 3) / 4, nz);
    k_sm121_j<<<grid, dim3(32, 4, 1), 0, stream>>>(out, scratch, plan->psn, plan->pwe, plan->i_lo, plan->i_hi,
                                                   plan->j_lo, plan->j_hi);
    if ((rc = check_launch("k_sm121_j"))) return rc;
    k_sm121_i<<<grid, dim3(32, 4, 1), 0, stream>>>(scratch, out, plan->psn, plan->pwe, plan->i_lo, plan->i_hi,
                                                   plan->j_lo, plan->j_hi);
    if ((rc = check_launch("k_sm121_i"))) return rc;
  }
  g_last_error.clear();
  return WRFGPU_OK;
}

extern "C" int wrfgpu_nest_rebuild_total(const double *parent_total, const double *parent_pert,
                                         const double *new_pert, size_t n, double *out_total, cudaStream_t stream) {
  if (parent_total == nullptr || parent_pert == nullptr || new_pert == nullptr || out_total == nullptr)
    return fail(WRFGPU_ERR_NULL_POINTER, "a total-rebuild pointer is NULL");
  if (n == 0) return WRFGPU_OK;
  k_nest_total<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(parent_total, parent_pert, new_pert, n, out_total);
  int rc = check_launch("k_nest_total");
  if (rc) return rc;
  g_last_error.clear();
  return WRFGPU_OK;
}

// ---------------------------------------------------------------------------
// Row copies of the y-slab decomposition (wrf_gpu_b200/sharding.py): rows of
// every level of (nz, ny, nx) arrays copied array to array (scatter / gather
// of a slab), or packed into / unpacked from one contiguous buffer (the halo
// blocks a rank sends and receives after each step).  One thread per element,
// consecutive threads along a row: coalesced on both sides.
// ---------------------------------------------------------------------------
namespace {
__global__ void k_copy_rows(const double *src, int src_ny, int src_j0, double *dst, int dst_ny, int dst_j0,
                            int nrows, int nx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  const int z = blockIdx.z;
  if (i >= nx) return;
  dst[((size_t)z * dst_ny + dst_j0 + r) * nx + i] = __ldg(src + ((size_t)z * src_ny + src_j0 + r) * nx + i);
}

struct RowBlocks {
  wrfgpu_row_block b[WRFGPU_MAX_ROW_BLOCKS];
};

constexpr int ROWS_THREADS = 256;

// Index space (chunks of ROWS_THREADS elements, blocks): element e of block
// blockIdx.y is (z, r, i) of its rows, at buffer[offset + e].
template <bool PACK>
__global__ void __launch_bounds__(ROWS_THREADS) k_rows_pack(RowBlocks B, double *buffer) {
  const wrfgpu_row_block &blk = B.b[blockIdx.y];
  const long long per_level = (long long)blk.nrows * blk.nx;
  const long long n = per_level * blk.nz;
  for (long long e = (long long)blockIdx.x * ROWS_THREADS + threadIdx.x; e < n;
       e += (long long)gridDim.x * ROWS_THREADS) {
    const long long z = e / per_level, rem = e - z * per_level;
    const long long r = rem / blk.nx, i = rem - r * blk.nx;
    const size_t f = ((size_t)z * blk.ny + blk.row0 + r) * blk.nx + i;
    if (PACK)
      buffer[blk.offset + e] = __ldg(blk.field + f);
    else
      blk.field[f] = __ldg(buffer + blk.offset + e);
  }
}

int rows_blocks(const wrfgpu_row_block *blocks, int nblocks, long long buffer_elems, RowBlocks &B, long long &most) {
  if (blocks == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "blocks is NULL");
  if (nblocks < 0 || nblocks > WRFGPU_MAX_ROW_BLOCKS) return fail(WRFGPU_ERR_BAD_SHAPE, "nblocks out of range");
  most = 0;
  for (int k = 0; k < nblocks; ++k) {
    const wrfgpu_row_block &b = blocks[k];
    if (b.field == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "a row block's field is NULL");
    if (b.nz < 1 || b.ny < 1 || b.nx < 1 || b.nrows < 0 || b.row0 < 0 || b.row0 + b.nrows > b.ny)
      return fail(WRFGPU_ERR_BAD_SHAPE, "a row block's rows lie outside its field");
    const long long n = (long long)b.nz * b.nrows * b.nx;
    if (b.offset < 0 || b.offset + n > buffer_elems)
      return fail(WRFGPU_ERR_BAD_SHAPE, "a row block lies outside the buffer");
    B.b[k] = b;
    most = n > most ? n : most;
  }
  return WRFGPU_OK;
}

template <bool PACK>
int rows_pack_impl(const wrfgpu_row_block *blocks, int nblocks, double *buffer, long long buffer_elems,
                   cudaStream_t stream) {
  if (buffer == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "buffer is NULL");
  RowBlocks B;
  long long most = 0;
  int rc = rows_blocks(blocks, nblocks, buffer_elems, B, most);
  if (rc) return rc;
  if (nblocks == 0 || most == 0) return WRFGPU_OK;
  long long chunks = (most + ROWS_THREADS - 1) / ROWS_THREADS;
  // a few elements per thread on large blocks; the grid stays a few waves of the SMs
  const long long cap = 148LL * 16;
  const int gx = (int)(chunks < cap ? chunks : cap);
  k_rows_pack<PACK><<<dim3(gx, nblocks), ROWS_THREADS, 0, stream>>>(B, buffer);
  rc = check_launch(PACK ? "k_rows_pack" : "k_rows_unpack");
  if (rc) return rc;
  g_last_error.clear();
  return WRFGPU_OK;
}
}  // namespace

extern "C" int wrfgpu_copy_rows(const double *src, int nz, int src_ny, int src_j0, double *dst, int dst_ny,
                                int dst_j0, int nrows, int nx, cudaStream_t stream) {
  if (src == nullptr || dst == nullptr) return fail(WRFGPU_ERR_NULL_POINTER, "src/dst is NULL");
  if (nz < 1 || nz > 65535 || nx < 1 || nrows < 0 || nrows > 65535 || src_ny < 1 || dst_ny < 1)
    return fail(WRFGPU_ERR_BAD_SHAPE, "bad row-copy extents");
  if (dst_j0 < 0 || dst_j0 + nrows > dst_ny || src_j0 < 0 || src_j0 + nrows > src_ny)
    return fail(WRFGPU_ERR_BAD_SHAPE, "rows out of range");
  if (nrows == 0) return WRFGPU_OK;
  k_copy_rows<<<dim3((nx + 127) / 128, nrows, nz), 128, 0, stream>>>(src, src_ny, src_j0, dst, dst_ny, dst_j0, nrows,
                                                                      nx);
  int rc = check_launch("k_copy_rows");
  if (rc) return rc;
  g_last_error.clear();
  return WRFGPU_OK;
}

extern "C" int wrfgpu_rows_pack(const wrfgpu_row_block *blocks, int nblocks, double *buffer,
                                long long buffer_elems, cudaStream_t stream) {
  return rows_pack_impl<true>(blocks, nblocks, buffer, buffer_elems, stream);
}

extern "C" int wrfgpu_rows_unpack(const wrfgpu_row_block *blocks, int nblocks, const double *buffer,
                                  long long buffer_elems, cudaStream_t stream) {
  return rows_pack_impl<false>(blocks, nblocks, const_cast<double *>(buffer), buffer_elems, stream);
}
