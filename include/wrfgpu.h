/*
 * wrfgpu.h -- C ABI of the B200-native split-explicit ARW RK3 dycore step.
 *
 * This replaces wrf_gpu's ``_rk_scan_step(carry, namelist, *, debug,
 * lead_seconds, physics_tendencies, capture_pre_halo)``
 * (src/gpuwrf/runtime/operational_mode.py:3319-3534): one full RK3 step --
 * flux-form advection, large-step PGF/Coriolis, small_step_prep, the acoustic
 * substep loop (advance_uv, advance_mu_t, advance_w with its tridiagonal
 * solve, calc_p_rho) and small_step_finish -- on device arrays.
 *
 * Conventions (the reference's data contract, contracts/state.py:82-206 and
 * contracts/grid.py:66-126):
 *   - every array is float64, C order (k, j, i), i fastest, contiguous;
 *   - u: (nz, ny, nx+1); v: (nz, ny+1, nx); w, ph, ww: (nz+1, ny, nx);
 *     mass fields: (nz, ny, nx); 2-D fields: (ny, nx);
 *   - map factors msfux/msfuy: (ny, nx+1); msfvx/msfvy: (ny+1, nx);
 *     msftx/msfty, f, e, sina, cosa: (ny, nx);
 *   - specified boundary strips u_bdy/v_bdy: (ntime, 4, width, nz, side_len)
 *     with sides W, E, S, N (contracts/state.py:96-106).
 *
 * Ownership: inputs are const device pointers, outputs caller-allocated
 * device pointers that must not alias any input; scratch is one
 * caller-provided workspace of wrfgpu_step_workspace_size() bytes.  Every
 * entry point takes a cudaStream_t and never synchronises, allocates or reads
 * device memory from the host, so a step can be captured in a CUDA graph.
 *
 * Errors: the reference raises at trace time for unsupported static
 * configurations (e.g. core/calc_p_rho.py:119-122); here every call returns
 * an int status, 0 on success, and wrfgpu_last_error_string() describes the
 * last failure of the calling thread.
 */
#ifndef WRFGPU_H
#define WRFGPU_H

#include <stddef.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WRFGPU_OK 0
#define WRFGPU_ERR_UNSUPPORTED_CONFIG 1
#define WRFGPU_ERR_BAD_SHAPE 2
#define WRFGPU_ERR_CUDA 3
#define WRFGPU_ERR_NULL_POINTER 4
#define WRFGPU_ERR_WORKSPACE 5

#define WRFGPU_PRECISION_FP64 0
#define WRFGPU_PRECISION_MIXED 1

#define WRFGPU_NMOIST 6 /* qv, qc, qr, qi, qs, qg (operational_mode.py:3095) */

/* Static step controls: the OperationalNamelist fields the step reads
 * (runtime/operational_mode.py:410-700).  Fill with wrfgpu_step_params_init()
 * first; its defaults equal the reference dataclass defaults. */
typedef struct wrfgpu_step_params {
  int nx, ny, nz;
  double dx, dy;               /* grid.projection.dx_m / dy_m */
  double dt;                   /* namelist.dt_s */
  int acoustic_substeps;       /* namelist.acoustic_substeps */
  double epssm;                /* namelist.epssm (0.1) */
  int top_lid;                 /* namelist.top_lid */
  int w_damping;               /* 0 | 1 */
  int damp_opt;                /* 0 | 3 */
  double dampcoef, zdamp;
  int hypsometric_opt;         /* 1 (linear) | 2 (log) */
  int h_sca_adv_order;         /* rhs_ph horizontal order; <= 2 supported */
  int scalar_adv_opt;          /* theta limiter: 0 | 1 (PD) | 2 (mono) */
  int moist_adv_opt;           /* moisture advection: 0 (off) | 1 | 2 */
  int run_boundary;            /* namelist.run_boundary */
  int bc_ideal;                /* grid.bc.source == "ideal" */
  int spec_zone, relax_zone;   /* boundary_config (1, 4) */
  double update_cadence_s;     /* boundary_config.update_cadence_s */
  double normal_bdy_relax_strength; /* <0 selects the reference default 20 */
  int moist_cqw;               /* GPUWRF_MOIST_CQW (default on) */
  int w_coriolis;              /* GPUWRF_W_CORIOLIS (default on) */
  int precision;               /* WRFGPU_PRECISION_FP64 | _MIXED */
  /* scalar metrics (DycoreMetrics.cf1/cf2/cf3/p_top) */
  double cf1, cf2, cf3, p_top;
  /* top-face extrapolation weights of the large-step PGF
   * (core/rk_addtend_dry.py:282-288): cfn = (0.5*dnw[nz-1] + dn[nz-1])/dn[nz-1],
   * cfn1 = -0.5*dnw[nz-1]/dn[nz-1] */
  double cfn, cfn1;
  /* Kernel tile shapes (no counterpart in the reference; results do not
   * depend on them): levels per block of the level-marching stencil kernels
   * (5, 10 or 25), level lanes of the column kernel (8, 13, 16 or 17) and
   * its columns per block (16 or 32); 0 selects the built-in defaults (10,
   * 17 and 32).  wrfgpu_autotune picks them per grid. */
  int march_levels;
  int column_lanes;
  int column_width;
  /* OperationalNamelist.specified_adv_degrade (operational_mode.py:460; default
   * off): with specified lateral BCs, WRF's tiered flux orders near the edges
   * and no horizontal advection of the outermost cells
   * (flux_advection.py:288-391). */
  int specified_adv_degrade;
  /* OperationalNamelist.specified_bdy_cadence (operational_mode.py:453;
   * default off): with specified lateral BCs and a forecast lead, WRF's
   * relax_bdy_dry tendencies in the relax zone (from the step-start state)
   * and the ring-0 pins of the tangential winds, mu, theta, ph and the
   * zero-gradient w every acoustic substep (operational_mode.py:1984-2041,
   * 2478-2530, 3085-3092; coupling/boundary_apply.py:1148-1340).  Needs the
   * theta_bdy / ph_bdy / mu_bdy strips. */
  int specified_bdy_cadence;
  /* BoundaryConfig.force_geopotential (coupling/boundary_apply.py:110;
   * default 1).  0 makes a run_boundary, non-ideal domain the nested child
   * (operational_mode.py:1247-1254): the same non-periodic advance_mu_t,
   * stage omega and order<=6 rhs_ph as a specified domain, with the
   * specified-only degradation and cadence off, and the three opt-in nested
   * forcings below (BoundaryConfig defaults 0, boundary_apply.py:142-144;
   * operational_mode.py:1906-1968):
   *   nested_ph_relax  relax-zone ph' tendency from the stage state toward
   *                    ph_bdy, coupled with c1f*mut+c2f, over msfty, added to
   *                    the stage ph tendency (boundary_apply.py:1045-1068);
   *   nested_w_relax   the same for w toward w_bdy into the stage rw
   *                    tendency (boundary_apply.py:1071-1087);
   *   nested_ph_spec   the ring-0 ph' pin to ph_bdy every acoustic substep
   *                    after advance_w (boundary_apply.py:1299-1340).
   * All three read the strips at the step's lead. */
  int force_geopotential;
  int nested_ph_relax;
  int nested_w_relax;
  int nested_ph_spec;
  /* 1: the step merges the caller's RK1-fixed physics tendencies
   * (_rk_scan_step's physics_tendencies, a DryPhysicsTendencies,
   * dynamics/core/rk_addtend_dry.py:103-124) into every RK stage's
   * tendencies as rk_addtend_dry does (rk_addtend_dry.py:490-546;
   * operational_mode.py:3062-3075); the bundle's arrays are the inputs'
   * physics pointers (NULL = zero).  0 (default): no bundle. */
  int physics;
  /* 6th-order numerical diffusion (diff_6th_opt, operational_mode.py:
   * 2870-2876; dynamics/explicit_diffusion.py:160-226): 0 (default) off, any
   * other value (the reference tests int(diff_6th_opt) != 0) adds the
   * monotonic filter of u, v, w, theta, coupled by their dry-air
   * mass, to every stage's tendencies with coefficient
   * diff_6th_factor * 0.015625 / (2 dt) (default factor 0.12). */
  int diff_6th_opt;
  double diff_6th_factor;
  /* Second-order explicit diffusion (operational_mode.py:2878-2960), added
   * to every stage's coupled u, v, w, theta tendencies after the 6th-order
   * filter:
   *   diff_opt = 1 with km_opt = 4: WRF's 2-D Smagorinsky horizontal
   *     diffusion on coordinate surfaces (the real-data default), eddy
   *     viscosity c_s^2 l^2 |D| capped at 10 l, l = sqrt(dx dy), heat
   *     diffusivity xkmh / prandtl (dynamics/explicit_diffusion.py:960-1365);
   *     c_s is OperationalNamelist.c_s (default 0.25);
   *   const_nu_m2_s > 0: constant-K diffusion in the mass-conservative flux
   *     form, horizontal and vertical (explicit_diffusion.py:282-331).
   * Other diff_opt / km_opt pairs select nothing in the reference except
   * diff_opt = 2 with km_opt 2, 3 or 5 (the TKE / 3-D Smagorinsky closures),
   * which are rejected as not built. */
  int diff_opt;
  int km_opt;
  double c_s;
  double const_nu_m2_s;
} wrfgpu_step_params;

/* DycoreMetrics device arrays (contracts/grid.py:66-126). */
typedef struct wrfgpu_metrics {
  const double *c1h, *c2h, *c3h, *c4h;      /* (nz)   */
  const double *c1f, *c2f, *c3f, *c4f;      /* (nz+1) */
  const double *dn, *dnw, *rdn, *rdnw, *fnm, *fnp; /* (nz) */
  const double *msftx, *msfty;              /* (ny, nx)   */
  const double *msfux, *msfuy;              /* (ny, nx+1) */
  const double *msfvx, *msfvy;              /* (ny+1, nx) */
  const double *f, *e, *sina, *cosa;        /* (ny, nx)   */
} wrfgpu_metrics;

/* Step inputs: the OperationalCarry leaves the step reads
 * (runtime/operational_state.py:30-127). */
typedef struct wrfgpu_step_inputs {
  const double *u, *v, *w, *theta;
  const double *p_total, *p_perturbation, *ph_total, *ph_perturbation;
  const double *mu_total, *mu_perturbation;
  const double *q[WRFGPU_NMOIST];   /* may be NULL (dry: treated as zero) */
  const double *mudf;               /* carry.mudf (ny, nx) */
  /* namelist.tendencies base leaves, NULL = zero (the reference default) */
  const double *base_u, *base_v, *base_w, *base_theta, *base_mu;
  /* specified lateral boundary strips; NULL unless run_boundary */
  const double *u_bdy, *v_bdy;
  int bdy_ntime, bdy_width, bdy_side_len;
  /* further strips the specified boundary cadence reads (NULL otherwise):
   * full theta (nz levels), ph' (nz+1 levels) and mu' (1 level), same
   * (ntime, 4, width, levels, side_len) layout */
  const double *theta_bdy, *ph_bdy, *mu_bdy;
  /* w strip (nz+1 levels) the nested w relaxation reads (NULL otherwise);
   * ph_bdy is also read by the nested ph' relaxation and pin */
  const double *w_bdy;
  /* DryPhysicsTendencies leaves (params.physics = 1; each NULL = zero):
   * ru_tendf (u-face), rv_tendf (v-face), rw_tendf, ph_tendf (nz+1), t_tendf,
   * h_diabatic (mass), mu_tendf (ny, nx), and the boundary tendencies added
   * at the first RK stage only, phys_u_save ... phys_t_save.  ph_tendf and
   * phys_ph_save enter no output: the ph tendency of this path is rhs_ph's
   * (operational_mode.py:3083-3084). */
  const double *ru_tendf, *rv_tendf, *rw_tendf, *ph_tendf, *t_tendf, *mu_tendf, *h_diabatic;
  const double *phys_u_save, *phys_v_save, *phys_w_save, *phys_ph_save, *phys_t_save;
} wrfgpu_step_inputs;

/* Step outputs: the returned OperationalCarry (operational_mode.py:2234-2265). */
typedef struct wrfgpu_step_outputs {
  double *u, *v, *w, *theta;
  double *p_total, *p_perturbation, *ph_total, *ph_perturbation;
  double *mu_total, *mu_perturbation;
  double *q[WRFGPU_NMOIST];         /* written when the input q is non-NULL */
  double *t_2ave, *ww, *mudf, *muave, *muts, *ph_tend;
  double *u_save, *v_save, *w_save, *t_save, *ph_save, *mu_save, *ww_save;
} wrfgpu_step_outputs;

/* Fill params with the reference defaults (no grid).  Replaces
 * OperationalNamelist defaults (runtime/operational_mode.py:410-700). */
int wrfgpu_step_params_init(wrfgpu_step_params *params);

/* Check params against what this build supports; 0 when supported.
 * Mirrors the reference's trace-time ValueError/NotImplementedError. */
int wrfgpu_step_params_validate(const wrfgpu_step_params *params);

/* Workspace bytes one wrfgpu_rk3_step call needs for these params. */
int wrfgpu_step_workspace_size(const wrfgpu_step_params *params, size_t *bytes);

/* One RK3 dycore step.  Replaces _rk_scan_step
 * (runtime/operational_mode.py:3319-3534).  lead_seconds is the forecast
 * clock at step start (NaN = None); it only selects the boundary strip time. */
int wrfgpu_rk3_step(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics,
                    const wrfgpu_step_inputs *in, const wrfgpu_step_outputs *out,
                    double lead_seconds, void *workspace, size_t workspace_bytes,
                    cudaStream_t stream);

/* One RK3 step with the forecast clock on the device: lead_seconds_dev points
 * to one double (seconds at step start, device memory) that the kernels
 * read when they interpolate boundary strips in time.  Replaces the same
 * _rk_scan_step call as it sits in the reference's jitted loop, where
 * lead_seconds is a traced value (runtime/operational_mode.py:4929-4945,
 * lead_seconds = step_index * dt inside fori_loop; interpolate_boundary_leaf
 * takes it as an array, coupling/boundary_apply.py:329-345).  The lead is
 * always present (the NaN = None form is wrfgpu_rk3_step's); results are
 * identical to wrfgpu_rk3_step with the same value on the host, and one
 * captured CUDA graph of this call can be replayed for successive steps by
 * updating the device value alone. */
int wrfgpu_rk3_step_device_lead(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics,
                                const wrfgpu_step_inputs *in, const wrfgpu_step_outputs *out,
                                const double *lead_seconds_dev, void *workspace, size_t workspace_bytes,
                                cudaStream_t stream);

/* Size of the workspace that the library itself holds for
 * wrfgpu_rk3_step_static_workspace: 32 MiB per GPU, reserved in every
 * process that loads the library, on every GPU it runs on, until exit. */
#define WRFGPU_STATIC_WORKSPACE_BYTES ((size_t)32 << 20)

/* One RK3 step, like wrfgpu_rk3_step, but with its scratch taken from a
 * fixed array the library holds on each GPU (WRFGPU_STATIC_WORKSPACE_BYTES)
 * instead of a caller workspace.  No counterpart in the reference: it is for
 * callers that cannot allocate device memory at all -- a host framework whose
 * own pool owns the GPU's memory (so a cudaMalloc of ours could fail or
 * fragment it), or a host model that calls one routine per step with a fixed
 * argument list and has nowhere to keep a workspace between calls.  It calls
 * no cudaMalloc/cudaFree and no allocating library routine.
 *   - Grids whose wrfgpu_step_workspace_size() exceeds
 *     WRFGPU_STATIC_WORKSPACE_BYTES are rejected with WRFGPU_ERR_WORKSPACE.
 *   - The first call on a GPU looks up the array's device address (with that
 *     GPU current); make that first call before any stream capture.  The
 *     address is kept for the life of the process and does not survive a
 *     cudaDeviceReset of that GPU: do not call this entry point on a device
 *     after resetting it.
 *   - Nothing in the array needs to start at zero: the step writes every
 *     scratch value before reading it, and clears or copies mudf itself.
 *   - Every call on one GPU shares the one array, which keeps the previous
 *     call's contents: calls that overlap on that GPU (other streams, other
 *     host threads) race and corrupt each other's results.  Order them on one
 *     stream, or use wrfgpu_rk3_step with separate workspaces. */
int wrfgpu_rk3_step_static_workspace(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics,
                                     const wrfgpu_step_inputs *in, const wrfgpu_step_outputs *out,
                                     double lead_seconds, cudaStream_t stream);

/* Advance n independent domains (ensemble members or nest levels, of any
 * sizes) by one RK3 step each: member m is wrfgpu_rk3_step(&params[m],
 * &metrics[m], &in[m], &out[m], lead_seconds[m], workspace[m],
 * workspace_bytes[m], .).  Members are forked onto a pool of library-owned
 * streams behind `stream` and joined back into it, so they run concurrently
 * and a capture of `stream` records them as parallel graph branches.  The
 * pool is created by the first call on a device; make that call before any
 * stream capture.  Replaces the reference's separate per-domain
 * _rk_scan_step calls (nests and ensemble members each call it). */
int wrfgpu_rk3_step_batched(int n, const wrfgpu_step_params *params, const wrfgpu_metrics *metrics,
                            const wrfgpu_step_inputs *in, const wrfgpu_step_outputs *out,
                            const double *lead_seconds, void *const *workspace, const size_t *workspace_bytes,
                            cudaStream_t stream);

/* Time the tile-shape candidates on this grid (each a few full steps from
 * `in` into `out`, which are overwritten) and write the fastest to
 * params->march_levels / column_lanes / column_width.  No counterpart in the
 * reference.  Synchronises `stream`; call it outside stream capture. */
int wrfgpu_autotune(wrfgpu_step_params *params, const wrfgpu_metrics *metrics, const wrfgpu_step_inputs *in,
                    const wrfgpu_step_outputs *out, void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* The plain h5/v3 flux-form scalar advection operator on its own: tend =
 * L(ru, rv, rom) q for one field q (nz, ny, nx), doubly periodic, with the
 * transport velocities ru, rv (nz, ny, nx; west / south faces of each cell)
 * and rom (nz+1, ny, nx) held fixed.  Replaces advect_scalar_flux
 * (dynamics/flux_advection.py:482-568).  Uses params nx, ny, nz, dx, dy and
 * metrics msftx, rdnw, fnm, fnp. */
int wrfgpu_scalar_advection(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics, const double *q,
                            const double *ru, const double *rv, const double *rom, double *tend,
                            cudaStream_t stream);

/* Its adjoint with respect to q: q_bar = L^T tend_bar (the vector-Jacobian
 * product of wrfgpu_scalar_advection for fixed velocities).  No counterpart in
 * the reference, which has no differentiation. */
int wrfgpu_scalar_advection_adjoint(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics,
                                    const double *tend_bar, const double *ru, const double *rv, const double *rom,
                                    double *q_bar, cudaStream_t stream);

/* The full vector-Jacobian product at (q, ru, rv, rom): q_bar (as
 * wrfgpu_scalar_advection_adjoint) and the velocities' cotangents ru_bar,
 * rv_bar (nz, ny, nx) and rom_bar (nz+1, ny, nx; zero on the bottom and top
 * faces), so that <tend_bar, dL> = <q_bar, dq> + <ru_bar, d ru> +
 * <rv_bar, d rv> + <rom_bar, d rom>, the upwind switches held at their
 * forward sign (the operator is bilinear in q and the velocities away from
 * zero velocities).  One launch; any output may be NULL (not computed), not
 * all four. */
int wrfgpu_scalar_advection_vjp(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics, const double *q,
                                const double *tend_bar, const double *ru, const double *rv, const double *rom,
                                double *q_bar, double *ru_bar, double *rv_bar, double *rom_bar, cudaStream_t stream);

/* The same flux-form operator with its map-factor weights given: tend =
 * -hfac rdx (Fx(i+1) - Fx(i)) - hfac rdy (Fy(j+1) - Fy(j)) + vfac (-rdnw
 * (Fz(k+1) - Fz(k))) for a field q (nz, ny, nx) doubly periodic on its own
 * extent, hfac and vfac (ny, nx).  hfac NULL is metrics->msftx and vfac NULL
 * is 1 (wrfgpu_scalar_advection).  The periodic momentum advection is this
 * operator on the core faces with face-averaged transport velocities:
 * advect_u_flux (dynamics/flux_advection.py:1131-1202) with hfac = msfux and
 * vfac NULL, advect_v_flux (:1205-1274) with hfac = msfvy and vfac = msfvy /
 * msfvx, the averages and the wrap face formed by the caller. */
int wrfgpu_flux_advection(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics, const double *q,
                          const double *ru, const double *rv, const double *rom, const double *hfac,
                          const double *vfac, double *tend, cudaStream_t stream);

/* Its vector-Jacobian product (as wrfgpu_scalar_advection_vjp, with the same
 * hfac / vfac); q may be NULL when only q_bar is asked for.  In both, rom
 * NULL leaves the vertical flux out (the horizontal part of w's advection,
 * params.nz then being w's level count). */
int wrfgpu_flux_advection_vjp(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics, const double *q,
                              const double *tend_bar, const double *ru, const double *rv, const double *rom,
                              const double *hfac, const double *vfac, double *q_bar, double *ru_bar,
                              double *rv_bar, double *rom_bar, cudaStream_t stream);

/* The vertical flux divergence of w (nz+1, ny, nx) by the omega rom
 * (nz+1, ny, nx): advect_w_flux's _vdiv_w part (dynamics/flux_advection.py:
 * 1410-1482; the horizontal part is wrfgpu_flux_advection on w's levels with
 * the velocities interpolated to them and rom NULL).  Reads params nx, ny,
 * nz (mass levels), top_lid and metrics rdn. */
int wrfgpu_w_vertical_advection(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics, const double *w,
                                const double *rom, double *tend, cudaStream_t stream);

/* Its vector-Jacobian product: w_bar and rom_bar (either may be NULL) for a
 * cotangent tend_bar, the upwind switches held at their forward signs. */
int wrfgpu_w_vertical_advection_vjp(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics,
                                    const double *w, const double *rom, const double *tend_bar, double *w_bar,
                                    double *rom_bar, cudaStream_t stream);

/* One acoustic small step on its own (the reference's acoustic_substep_core,
 * core/acoustic.py:837-1150: advance_uv, advance_mu_t, advance_w with its
 * Thomas solve, calc_p_rho with smdiv memory), over the evolving work state of
 * AcousticCoreState (core/acoustic.py:112-292) with the stage constants held
 * fixed.  Layouts as the step's: u (nz, ny, nx+1), v (nz, ny+1, nx); w, ph, ww
 * (nz+1, ny, nx); theta_w, t_2ave, p, pm1, al and the stage 3-D constants
 * (nz, ny, nx), except rw_tend, ph_tend, cqw, pt1, a, alpha, gamma, ww_1 and
 * w_save (nz+1, ny, nx); 2-D fields (ny, nx); cqu / u_tend / u_1 u-face, cqv /
 * v_tend / v_1 v-face shaped. */
typedef struct wrfgpu_acoustic_work {
  double *u, *v, *w, *ph, *theta_w, *t_2ave, *p, *pm1, *al, *ww; /* 3-D */
  double *mu, *muts, *muave, *mudf;                              /* 2-D */
} wrfgpu_acoustic_work;

typedef struct wrfgpu_acoustic_consts {
  const double *u_tend, *v_tend, *t_tend, *rw_tend, *ph_tend; /* stage tendencies */
  const double *alt, *pb, *c2a, *cqu, *cqv, *cqw, *php;       /* stage diagnostics */
  const double *pt1;                                          /* ph_1 + phb (faces) */
  const double *a, *alpha, *gamma;                            /* calc_coef_w */
  const double *ww_1;                                         /* stage omega */
  const double *mut, *muu, *muv;                              /* stage masses */
  const double *mu_tend;                                      /* NULL = zero */
  const double *u_1, *v_1, *w_save, *theta;                   /* stage u, v, w, theta */
  const double *phb0;                                         /* base geopotential, face 0 (ny, nx) */
  /* run_boundary: the stage's normal-wind work targets, u- / v-face shaped
   * (coupling/boundary_apply.py:729-781), blended into the relax zone every
   * substep; NULL otherwise */
  const double *u_target, *v_target;
} wrfgpu_acoustic_consts;

/* Scratch bytes of wrfgpu_acoustic_substep / _vjp for these params. */
int wrfgpu_acoustic_workspace_size(const wrfgpu_step_params *params, size_t *bytes);

/* x <- one acoustic substep of length dts from x (in place), on doubly
 * periodic or specified / nested domains (the boundary relaxation toward
 * u_target / v_target, advance_mu_t's frozen ring and drain limiter), without
 * the boundary cadence's ring-0 pins and without the w_damping CFL term. */
int wrfgpu_acoustic_substep(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics,
                            const wrfgpu_acoustic_consts *consts, wrfgpu_acoustic_work *x, double dts,
                            void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* Cotangents of the stage tendencies the substep reads (wrfgpu_acoustic_consts
 * u_tend .. ph_tend, mu_tend), shaped like them; a NULL member is not
 * computed. */
typedef struct wrfgpu_acoustic_tend_cot {
  double *u_tend, *v_tend, *t_tend, *rw_tend, *ph_tend, *mu_tend;
} wrfgpu_acoustic_tend_cot;

/* Its vector-Jacobian product at x: cot_in = J(x)^T cot_out, J the Jacobian of
 * wrfgpu_acoustic_substep with respect to the work state, constants fixed
 * and the drain limiter's scale held at its forward value (muave enters no
 * output of an updated column: its cot_in is zero there).  x_out is the substep's
 * output from x (a stored checkpoint); NULL recomputes it into the
 * workspace.  cot_tend (may be NULL) receives the cotangents of the stage
 * tendencies.  cot_out is read only; cot_in must not alias it.  No
 * counterpart in the reference, which has no differentiation. */
int wrfgpu_acoustic_substep_vjp(const wrfgpu_step_params *params, const wrfgpu_metrics *metrics,
                                const wrfgpu_acoustic_consts *consts, const wrfgpu_acoustic_work *x,
                                const wrfgpu_acoustic_work *x_out, const wrfgpu_acoustic_work *cot_out,
                                wrfgpu_acoustic_work *cot_in, wrfgpu_acoustic_tend_cot *cot_tend, double dts,
                                void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* Boundary strips of the end-of-step lateral boundary pass, each
 * (ntime, 4, width, levels, side_len) like u_bdy (sides W, E, S, N): u, v,
 * theta, the six moisture species (nz levels), w, ph' and phb (nz+1), p' and
 * pb (nz), mu' and mub (1 level).  A NULL moisture strip leaves that species
 * untouched. */
typedef struct wrfgpu_lbc_leaves {
  const double *u, *v, *w, *theta;
  const double *q[WRFGPU_NMOIST];
  const double *p, *pb, *mu, *mub, *ph, *phb;
  int ntime, width, side_len;
} wrfgpu_lbc_leaves;

/* The end-of-step lateral boundary pass of a forecast step, replacing
 * apply_lateral_boundaries(state, lead_seconds, dt_s, boundary_config,
 * metrics, dry_spec_only=...) (coupling/boundary_apply.py:170-326): the
 * state `in` (its 10 state leaves and moisture) with the strips at
 * lead_seconds into `out` (the same leaves; out's carry pointers are not
 * used; out must not alias in).  Full pass: u, v, w, theta, p', pb, mu', mub
 * and (params.force_geopotential) ph', phb relaxed in the relax zone and set
 * in the outer row (totals rebuilt as base + perturbation), moisture relaxed
 * and clipped at zero.  dry_spec_only = 1 (the specified boundary cadence's
 * pass): u, v, theta, mu', mub, ph', phb set in the outer row only, w and p
 * untouched, moisture as in the full pass.  Reads params nx, ny, nz, dt,
 * update_cadence_s, spec_zone = 1, relax_zone = 4, force_geopotential. */
int wrfgpu_apply_lateral_boundaries(const wrfgpu_step_params *params, const wrfgpu_step_inputs *in,
                                    const wrfgpu_lbc_leaves *leaves, const wrfgpu_step_outputs *out,
                                    double lead_seconds, int dry_spec_only, cudaStream_t stream);

/* The theta limiter's record (the dict of
 * _positive_definite_theta_increment_limiter, runtime/operational_mode.py:
 * 1444-1454): offending cells, the first one as [x, y, z] ([-1, -1, -1] when
 * none), and the mass-weighted theta integral before and after. */
typedef struct wrfgpu_theta_limiter_diag {
  int limited_cell_count;
  int first_limited_cell_xyz[3];
  double mass_before, mass_after, mass_residual;
} wrfgpu_theta_limiter_diag;

/* Workspace bytes of wrfgpu_step_epilogue for these params. */
int wrfgpu_step_epilogue_workspace_size(const wrfgpu_step_params *params, size_t *bytes);

/* The forecast step after _rk_scan_step, without physics, replacing
 * runtime/operational_mode.py:4950-4983 of
 * _physics_boundary_step_with_limiter_diagnostics: `next` is the step's
 * output state, `origin` the step-start state (physical_origin), `out` the
 * new state (must not alias `next` or `origin`).
 * Guards on (disable_guards = 0): the theta increment limiter weighted by
 * next's mu_total, the dry-mass guard and the mixing-ratio guard of every
 * moisture species against origin (_limit_guarded_dynamics_state_with_
 * diagnostics, _valid_mixing_ratio); then, when params.run_boundary, the
 * end-of-step boundary pass (as wrfgpu_apply_lateral_boundaries, with
 * dry_spec_only = the specified boundary cadence is active) followed by the
 * finite guard of u, v, w, theta, p, p', ph, ph', the mixing-ratio guard of
 * qv and the dry-mass guard, all against origin.  Guards off: the boundary
 * pass alone (or a copy).  `leaves` is read only when params.run_boundary.
 * `diag` (device memory, may be NULL) receives the limiter's record (the
 * empty record with guards off).  Enqueued on `stream`; allocates nothing. */
int wrfgpu_step_epilogue(const wrfgpu_step_params *params, const wrfgpu_step_inputs *origin,
                         const wrfgpu_step_inputs *next, const wrfgpu_lbc_leaves *leaves,
                         const wrfgpu_step_outputs *out, double lead_seconds, int disable_guards,
                         wrfgpu_theta_limiter_diag *diag, void *workspace, size_t workspace_bytes,
                         cudaStream_t stream);

/* wrfgpu_step_epilogue with the forecast clock on the device (one double at
 * lead_seconds_dev, seconds), read by the boundary pass's kernels: the
 * reference passes the traced lead_seconds of its jitted loop to
 * apply_lateral_boundaries (runtime/operational_mode.py:4966-4969).  Results
 * are identical to wrfgpu_step_epilogue with the same value on the host. */
int wrfgpu_step_epilogue_device_lead(const wrfgpu_step_params *params, const wrfgpu_step_inputs *origin,
                                     const wrfgpu_step_inputs *next, const wrfgpu_lbc_leaves *leaves,
                                     const wrfgpu_step_outputs *out, const double *lead_seconds_dev,
                                     int disable_guards, wrfgpu_theta_limiter_diag *diag, void *workspace,
                                     size_t workspace_bytes, cudaStream_t stream);

/* ------------------------------------------------------------------------
 * Nest coupling around the step (a nested child's boundary leaves from its
 * parent, and the child's feedback onto the parent).
 * ------------------------------------------------------------------------ */

/* Static parent -> child bilinear gather of one staggering (device arrays):
 * per child row the floor / ceil parent rows y0, y1 and the weight wy toward
 * y1, per child column x0, x1, wx (nesting/interp.py:68-190, built on the host
 * with the WRF sint cell-centered or the node-aligned registration). */
typedef struct wrfgpu_nest_interp {
  const int *y0, *y1, *x0, *x1;   /* (child_ny), (child_nx) */
  const double *wy, *wx;
  int child_ny, child_nx;         /* child extent of this staggering */
  int parent_ny, parent_nx;       /* parent extent of this staggering */
} wrfgpu_nest_interp;

/* A parent field (nz, parent_ny, parent_nx) interpolated onto the whole child
 * grid (nz, child_ny, child_nx): rows first, then columns.  Replaces
 * interp_sint_linear / interp_bilinear (nesting/interp.py:248-314) and
 * interp_parent_field_to_child (nesting/boundary_construction.py:454-468). */
int wrfgpu_nest_interp_field(const wrfgpu_nest_interp *w, const double *parent, int nz, double *child_out,
                             cudaStream_t stream);

/* One two-time child boundary leaf (2, 4, width, leaf_z, leaf_side): time 0
 * the child field's own ring (with child_sub set: of child - child_sub, a
 * base state from a total and its perturbation), time 1 the parent
 * interpolated to the same ring cells (w = NULL: the time-0 ring again, as
 * for the base leaves); W / E
 * columns and S / N rows from the domain edge inward, zero beyond the field's
 * extent (side_len = the strips' tangential length) or the leaf's.  One call
 * per leaf replaces build_child_boundary_package
 * (nesting/boundary_construction.py:360-451: field_sides_3d/_2d, _fit and the
 * two-time stack). */
int wrfgpu_nest_ring_leaf(const wrfgpu_nest_interp *w, const double *parent, const double *child,
                          const double *child_sub, int nz, int child_ny, int child_nx, int width, int side_len,
                          int leaf_z, int leaf_side, double *leaf, cudaStream_t stream);

/* WRF copy_fcn feedback plan of one staggering (device index arrays) and its
 * sm121 smoother interior (coupling/boundary_feedback.py:170-319). */
typedef struct wrfgpu_nest_feedback_plan {
  const int *parent_lin;          /* (npts) parent linear index in a (psn, pwe) plane */
  const int *child_lin;           /* (npts, stencil) child donors in a (csn, cwe) plane */
  int npts, stencil, pwe, psn, cwe, csn;
  int i_lo, i_hi, j_lo, j_hi;     /* sm121 interior, 0-based half-open */
  int smooth;                     /* smooth_option != 0 */
} wrfgpu_nest_feedback_plan;

/* out = parent with the overlap points set to the mean of their child donors,
 * then (plan->smooth) the sm121 1-2-1 smoother over the interior; nz levels
 * of (psn, pwe); scratch is one field of the same size (used by the
 * smoother); out may alias parent.  Replaces apply_feedback + sm121_smooth
 * (coupling/boundary_feedback.py:400-494). */
int wrfgpu_nest_feedback(const wrfgpu_nest_feedback_plan *plan, const double *parent, const double *child, int nz,
                         double *out, double *scratch, cudaStream_t stream);

/* out_total = (parent_total - parent_pert) + new_pert over n elements: the
 * totals rebuilt after feedback (coupling/boundary_feedback.py:557-568). */
int wrfgpu_nest_rebuild_total(const double *parent_total, const double *parent_pert, const double *new_pert,
                              size_t n, double *out_total, cudaStream_t stream);

/* ---- y-slab decomposition: row copies ------------------------------------
 * The multi-GPU form of the step (wrf_gpu_b200/sharding.py) gives each rank
 * a slab of rows plus halo rows and, after each step, exchanges the halo
 * blocks of the fields the next step reads.  These entries move those rows;
 * they replace the reference's x-halo refresh by lax.ppermute
 * (runtime/sharding.py:800-866) and its partition / merge of the state
 * (runtime/sharding.py:515-590, 768-798). */

/* Rows [src_j0, src_j0 + nrows) of every level of src (nz, src_ny, nx) copied
 * into rows [dst_j0, dst_j0 + nrows) of dst (nz, dst_ny, nx). */
int wrfgpu_copy_rows(const double *src, int nz, int src_ny, int src_j0, double *dst, int dst_ny, int dst_j0,
                     int nrows, int nx, cudaStream_t stream);

/* One block of rows of one array: rows [row0, row0 + nrows) of every level
 * of field (nz, ny, nx), stored in a packed buffer from element offset on as
 * (nz, nrows, nx). */
typedef struct wrfgpu_row_block {
  double *field;
  int nz, ny, nx;
  int row0, nrows;
  long long offset;
} wrfgpu_row_block;

#define WRFGPU_MAX_ROW_BLOCKS 40

/* Every block's rows copied into buffer (buffer_elems doubles), one launch. */
int wrfgpu_rows_pack(const wrfgpu_row_block *blocks, int nblocks, double *buffer, long long buffer_elems,
                     cudaStream_t stream);

/* The inverse: every block's rows written from buffer, one launch. */
int wrfgpu_rows_unpack(const wrfgpu_row_block *blocks, int nblocks, const double *buffer, long long buffer_elems,
                       cudaStream_t stream);

/* Number of kernel launches one wrfgpu_rk3_step issues for these params. */
int wrfgpu_step_launch_count(const wrfgpu_step_params *params, int *launches);

/* Per-kernel device timing (no counterpart in the reference: its XLA program
 * is profiled with nsys).  When enabled, every launch of wrfgpu_rk3_step is
 * bracketed by CUDA events from a pool of max_records pairs;
 * wrfgpu_profile_read synchronises on the last event, returns the summed
 * milliseconds and launch counts per kernel class and resets the pool.
 * Not for use inside CUDA graph capture. */
int wrfgpu_profile_enable(int enable, int max_records);
int wrfgpu_profile_read(double *total_ms, int *counts, int nclasses, int *dropped);
int wrfgpu_profile_class_count(void);
const char *wrfgpu_profile_class_name(int cls);

/* Last error of the calling host thread ("" when none). */
const char *wrfgpu_last_error_string(void);

/* Library version string. */
const char *wrfgpu_version(void);

#ifdef __cplusplus
}
#endif

#endif /* WRFGPU_H */
