"""Host-side mirror of wrf_gpu's RK3 dycore step interface, on the CUDA C ABI.

``rk_scan_step(carry, namelist, *, debug, lead_seconds, physics_tendencies,
capture_pre_halo)`` keeps the signature of the reference's ``_rk_scan_step``
(``src/gpuwrf/runtime/operational_mode.py:3319-3327``) and returns a new
``OperationalCarry`` (functional, like the reference).  The data types mirror
``State`` (``contracts/state.py:82-206``), ``DycoreMetrics``
(``contracts/grid.py:66-126``), ``OperationalCarry``
(``runtime/operational_state.py:30-127``) and the ``OperationalNamelist``
fields the step reads (``runtime/operational_mode.py:410-700``), with torch
float64 CUDA tensors as leaves.  PyTorch only provides device memory and the
current stream; all arithmetic runs in ``libwrfgpu.so``.

Unsupported static configurations raise ``NotImplementedError`` before any
launch, as the reference raises at trace time.
"""

from __future__ import annotations

import ctypes
import math
from collections import OrderedDict
from dataclasses import dataclass, field, fields, replace
from typing import Any

import numpy as np
import torch

from . import _capi

MOIST = ("qv", "qc", "qr", "qi", "qs", "qg")
STATE_FIELDS = _capi.STATE_FIELDS
_LEAVES = ("u_bdy", "v_bdy", "theta_bdy", "ph_bdy", "mu_bdy", "w_bdy", "qv_bdy", "qc_bdy", "qr_bdy", "qi_bdy",
           "qs_bdy", "qg_bdy", "p_bdy", "pb_bdy", "mub_bdy", "phb_bdy")
CARRY_FIELDS = _capi.CARRY_OUT_FIELDS
METRIC_ARRAYS = _capi.METRIC_FIELDS


def _dev(x, device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(np.asarray(x, dtype=np.float64)), device=device)


def _ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if t.dtype != torch.float64 or not t.is_contiguous() or not t.is_cuda:
        raise ValueError("wrf_gpu_b200 arrays must be contiguous float64 CUDA tensors")
    return t.data_ptr()


@dataclass
class DycoreMetrics:
    """``DycoreMetrics`` leaves on the device (contracts/grid.py:66-126)."""

    c1h: torch.Tensor
    c2h: torch.Tensor
    c3h: torch.Tensor
    c4h: torch.Tensor
    c1f: torch.Tensor
    c2f: torch.Tensor
    c3f: torch.Tensor
    c4f: torch.Tensor
    dn: torch.Tensor
    dnw: torch.Tensor
    rdn: torch.Tensor
    rdnw: torch.Tensor
    fnm: torch.Tensor
    fnp: torch.Tensor
    msftx: torch.Tensor
    msfty: torch.Tensor
    msfux: torch.Tensor
    msfuy: torch.Tensor
    msfvx: torch.Tensor
    msfvy: torch.Tensor
    f: torch.Tensor
    e: torch.Tensor
    sina: torch.Tensor
    cosa: torch.Tensor
    cf1: float
    cf2: float
    cf3: float
    p_top: float

    @classmethod
    def from_host(cls, m, device="cuda") -> "DycoreMetrics":
        kw = {n: _dev(getattr(m, n), device) for n in METRIC_ARRAYS}
        return cls(**kw, cf1=float(m.cf1), cf2=float(m.cf2), cf3=float(m.cf3), p_top=float(m.p_top))

    def cfn(self) -> tuple[float, float]:
        """Top-face weights of the large-step PGF (core/rk_addtend_dry.py:282-288)."""
        dn_top = float(self.dn[-1].item())
        dnw_top = float(self.dnw[-1].item())
        dn_safe = dn_top if abs(dn_top) > 1.0e-30 else 1.0
        return (0.5 * dnw_top + dn_top) / dn_safe, -0.5 * dnw_top / dn_safe


@dataclass
class State:
    """The ``State`` leaves the step reads and writes (contracts/state.py:82-206)."""

    u: torch.Tensor
    v: torch.Tensor
    w: torch.Tensor
    theta: torch.Tensor
    p_total: torch.Tensor
    p_perturbation: torch.Tensor
    ph_total: torch.Tensor
    ph_perturbation: torch.Tensor
    mu_total: torch.Tensor
    mu_perturbation: torch.Tensor
    qv: torch.Tensor | None = None
    qc: torch.Tensor | None = None
    qr: torch.Tensor | None = None
    qi: torch.Tensor | None = None
    qs: torch.Tensor | None = None
    qg: torch.Tensor | None = None
    u_bdy: torch.Tensor | None = None
    v_bdy: torch.Tensor | None = None
    theta_bdy: torch.Tensor | None = None
    ph_bdy: torch.Tensor | None = None
    mu_bdy: torch.Tensor | None = None
    w_bdy: torch.Tensor | None = None
    # further strips of the end-of-step lateral boundary pass
    qv_bdy: torch.Tensor | None = None
    qc_bdy: torch.Tensor | None = None
    qr_bdy: torch.Tensor | None = None
    qi_bdy: torch.Tensor | None = None
    qs_bdy: torch.Tensor | None = None
    qg_bdy: torch.Tensor | None = None
    p_bdy: torch.Tensor | None = None
    pb_bdy: torch.Tensor | None = None
    mub_bdy: torch.Tensor | None = None
    phb_bdy: torch.Tensor | None = None

    @property
    def p(self):
        return self.p_total

    @property
    def ph(self):
        return self.ph_total

    @property
    def mu(self):
        return self.mu_total

    def replace(self, **kw) -> "State":
        return replace(self, **kw)

    @classmethod
    def from_host(cls, s, device="cuda") -> "State":
        kw = {}
        for f_ in fields(cls):
            v = getattr(s, f_.name, None)
            kw[f_.name] = None if v is None else _dev(v, device)
        return cls(**kw)

    def to_host(self) -> dict:
        return {f_.name: getattr(self, f_.name).cpu().numpy() for f_ in fields(self)
                if getattr(self, f_.name) is not None}


@dataclass
class OperationalCarry:
    """``OperationalCarry`` (runtime/operational_state.py:30-127), dycore leaves only."""

    state: State
    t_2ave: torch.Tensor | None = None
    ww: torch.Tensor | None = None
    mudf: torch.Tensor | None = None
    muave: torch.Tensor | None = None
    muts: torch.Tensor | None = None
    ph_tend: torch.Tensor | None = None
    u_save: torch.Tensor | None = None
    v_save: torch.Tensor | None = None
    w_save: torch.Tensor | None = None
    t_save: torch.Tensor | None = None
    ph_save: torch.Tensor | None = None
    mu_save: torch.Tensor | None = None
    ww_save: torch.Tensor | None = None
    base_state: Any = None

    def replace(self, **kw) -> "OperationalCarry":
        return replace(self, **kw)


def initial_operational_carry(state: State) -> OperationalCarry:
    """``initial_operational_carry`` (runtime/operational_state.py:141-211), dycore leaves."""
    ny, nx = state.mu_total.shape
    z = lambda t: torch.zeros_like(t)
    return OperationalCarry(
        state=state, t_2ave=z(state.theta), ww=z(state.w), mudf=z(state.mu_total), muave=z(state.mu_total),
        muts=state.mu_total.clone(), ph_tend=z(state.ph_perturbation), u_save=state.u.clone(),
        v_save=state.v.clone(), w_save=state.w.clone(), t_save=state.theta.clone(),
        ph_save=state.ph_perturbation.clone(), mu_save=state.mu_perturbation.clone(), ww_save=z(state.w))


@dataclass
class Tendencies:
    """``namelist.tendencies`` base leaves (contracts/state.py Tendencies); None = zero."""

    u: torch.Tensor | None = None
    v: torch.Tensor | None = None
    w: torch.Tensor | None = None
    theta: torch.Tensor | None = None
    mu: torch.Tensor | None = None


@dataclass
class BoundaryConfig:
    """``BoundaryConfig`` (coupling/boundary_apply.py:71-151) fields the step reads."""

    spec_bdy_width: int = 5
    spec_zone: int = 1
    relax_zone: int = 4
    update_cadence_s: float = 3600.0
    force_geopotential: bool = True
    nested_ph_relax: bool = False
    nested_w_relax: bool = False
    nested_ph_spec: bool = False
    normal_bdy_relax_strength: float | None = None


@dataclass
class OperationalNamelist:
    """The ``OperationalNamelist`` controls the RK3 step reads
    (runtime/operational_mode.py:410-700).  Defaults are the reference's."""

    metrics: DycoreMetrics
    nx: int
    ny: int
    nz: int
    dx_m: float
    dy_m: float
    tendencies: Tendencies = field(default_factory=Tendencies)
    dt_s: float = 10.0
    acoustic_substeps: int = 10
    rk_order: int = 3
    epssm: float = 0.1
    hypsometric_opt: int = 1
    h_sca_adv_order: int = 2
    specified_bdy_cadence: bool = False
    specified_adv_degrade: bool = False
    top_lid: bool = False
    run_physics: bool = True
    run_boundary: bool = True
    bc_source: str = "ideal"
    disable_guards: bool = False
    boundary_config: BoundaryConfig = field(default_factory=BoundaryConfig)
    use_vertical_solver: bool = True
    w_damping: int = 0
    damp_opt: int = 0
    dampcoef: float = 0.0
    zdamp: float = 5000.0
    diff_opt: int = 0
    km_opt: int = 0
    diff_6th_opt: int = 0
    diff_6th_factor: float = 0.12
    c_s: float = 0.25
    const_nu_m2_s: float = 0.0
    use_deformation_momentum_diffusion: bool = False
    use_flux_advection: bool = False
    scalar_adv_opt: int = 0
    moist_adv_opt: int = 0
    mp_physics: int = 8
    acoustic_precision_mode: str = "fp64_default"
    moist_cqw: bool = True
    w_coriolis: bool = True
    precision: str = "fp64"

    @classmethod
    def from_case(cls, case, metrics: DycoreMetrics | None = None, device="cuda", **overrides) -> "OperationalNamelist":
        c = case.controls
        m = metrics if metrics is not None else DycoreMetrics.from_host(case.metrics, device)
        bc = BoundaryConfig(spec_zone=c["spec_zone"], relax_zone=c["relax_zone"],
                            update_cadence_s=c["update_cadence_s"],
                            normal_bdy_relax_strength=c["normal_bdy_relax_strength"],
                            force_geopotential=bool(c.get("force_geopotential", True)),
                            nested_ph_relax=bool(c.get("nested_ph_relax", False)),
                            nested_w_relax=bool(c.get("nested_w_relax", False)),
                            nested_ph_spec=bool(c.get("nested_ph_spec", False)))
        kw = dict(metrics=m, nx=case.nx, ny=case.ny, nz=case.nz, dx_m=c["dx"], dy_m=c["dy"], dt_s=c["dt_s"],
                  acoustic_substeps=c["acoustic_substeps"], epssm=c["epssm"], hypsometric_opt=c["hypsometric_opt"],
                  h_sca_adv_order=c["h_sca_adv_order"], top_lid=c["top_lid"], run_physics=False,
                  run_boundary=c["run_boundary"], bc_source="ideal" if c["bc_ideal"] else "wrfbdy",
                  boundary_config=bc, w_damping=c["w_damping"], damp_opt=c["damp_opt"], dampcoef=c["dampcoef"],
                  zdamp=c["zdamp"], use_flux_advection=True, scalar_adv_opt=c["scalar_adv_opt"],
                  moist_adv_opt=c["moist_adv_opt"], moist_cqw=c["moist_cqw"], w_coriolis=c["w_coriolis"],
                  specified_adv_degrade=bool(c.get("specified_adv_degrade", False)),
                  specified_bdy_cadence=bool(c.get("specified_bdy_cadence", False)),
                  diff_6th_opt=int(c.get("diff_6th_opt", 0)), diff_6th_factor=float(c.get("diff_6th_factor", 0.12)),
                  diff_opt=int(c.get("diff_opt", 0)), km_opt=int(c.get("km_opt", 0)), c_s=float(c.get("c_s", 0.25)),
                  const_nu_m2_s=float(c.get("const_nu_m2_s", 0.0)))
        kw.update(overrides)
        return cls(**kw)


def _unsupported(nl: OperationalNamelist, physics_tendencies) -> str | None:
    if not nl.use_flux_advection:
        return "use_flux_advection=False (primitive M4 advection path) is not built"
    if not nl.use_vertical_solver:
        return "use_vertical_solver=False is not built"
    if nl.rk_order != 3:
        return "rk_order must be 3"
    if int(nl.diff_opt) == 2 and int(nl.km_opt) in (2, 3, 5):
        return "diff_opt=2 with km_opt 2/3/5 (TKE / 3-D Smagorinsky closures) is not built"
    if nl.const_nu_m2_s > 0.0 and nl.use_deformation_momentum_diffusion:
        return "the deformation-tensor momentum form of the constant-K diffusion is not built"
    if nl.moist_adv_opt and nl.mp_physics in (7, 17, 18, 19, 21, 22, 24, 26, 27, 28, 38):
        return "extra advected species of this mp_physics family are not built"
    if nl.acoustic_precision_mode != "fp64_default":
        return "acoustic_precision_mode other than fp64_default is not built"
    return None


def step_params(nl: OperationalNamelist) -> _capi.StepParams:
    lib = _capi.load()
    p = _capi.StepParams()
    _capi.check(lib.wrfgpu_step_params_init(ctypes.byref(p)))
    p.nx, p.ny, p.nz = nl.nx, nl.ny, nl.nz
    p.dx, p.dy, p.dt = nl.dx_m, nl.dy_m, nl.dt_s
    p.acoustic_substeps = nl.acoustic_substeps
    p.epssm = nl.epssm
    p.top_lid = int(bool(nl.top_lid))
    p.w_damping, p.damp_opt = int(nl.w_damping), int(nl.damp_opt)
    p.dampcoef, p.zdamp = float(nl.dampcoef), float(nl.zdamp)
    p.hypsometric_opt, p.h_sca_adv_order = int(nl.hypsometric_opt), int(nl.h_sca_adv_order)
    p.scalar_adv_opt, p.moist_adv_opt = int(nl.scalar_adv_opt), int(nl.moist_adv_opt)
    p.run_boundary = int(bool(nl.run_boundary))
    p.bc_ideal = int(nl.bc_source == "ideal")
    p.spec_zone, p.relax_zone = nl.boundary_config.spec_zone, nl.boundary_config.relax_zone
    p.update_cadence_s = float(nl.boundary_config.update_cadence_s)
    s = nl.boundary_config.normal_bdy_relax_strength
    p.normal_bdy_relax_strength = -1.0 if s is None else float(s)
    p.moist_cqw, p.w_coriolis = int(bool(nl.moist_cqw)), int(bool(nl.w_coriolis))
    p.precision = _capi.WRFGPU_PRECISION_MIXED if nl.precision == "mixed" else _capi.WRFGPU_PRECISION_FP64
    p.specified_adv_degrade = 1 if nl.specified_adv_degrade else 0
    p.specified_bdy_cadence = 1 if nl.specified_bdy_cadence else 0
    bc = nl.boundary_config
    p.force_geopotential = int(bool(bc.force_geopotential))
    p.nested_ph_relax, p.nested_w_relax = int(bool(bc.nested_ph_relax)), int(bool(bc.nested_w_relax))
    p.nested_ph_spec = int(bool(bc.nested_ph_spec))
    p.diff_6th_opt, p.diff_6th_factor = int(nl.diff_6th_opt), float(nl.diff_6th_factor)
    p.diff_opt, p.km_opt, p.c_s = int(nl.diff_opt), int(nl.km_opt), float(nl.c_s)
    p.const_nu_m2_s = float(nl.const_nu_m2_s)
    m = nl.metrics
    p.cf1, p.cf2, p.cf3, p.p_top = m.cf1, m.cf2, m.cf3, m.p_top
    p.cfn, p.cfn1 = m.cfn()
    return p


class Stepper:
    """Prepared step for one namelist: params, metrics struct, workspace."""

    def __init__(self, nl: OperationalNamelist, device="cuda", physics: bool = False, own_workspace: bool = True):
        reason = _unsupported(nl, None)
        if reason:
            raise NotImplementedError(reason)
        self.lib = _capi.load()
        self.nl = nl
        self.device = torch.device(device)
        self.params = step_params(nl)
        # a DryPhysicsTendencies bundle is merged into every stage (rk_addtend_dry)
        self.params.physics = 1 if physics else 0
        _capi.check(self.lib.wrfgpu_step_params_validate(ctypes.byref(self.params)))
        nbytes = ctypes.c_size_t(0)
        _capi.check(self.lib.wrfgpu_step_workspace_size(ctypes.byref(self.params), ctypes.byref(nbytes)))
        self.workspace_bytes = int(nbytes.value)
        # without an own workspace, every step_into takes one from torch's
        # caching allocator on the launching stream (stream-ordered reuse)
        self.workspace = (torch.empty(self.workspace_bytes, dtype=torch.uint8, device=device)
                          if own_workspace else None)
        self.metrics = _capi.Metrics(*[_ptr(getattr(nl.metrics, n)) for n in METRIC_ARRAYS])
        n = ctypes.c_int(0)
        _capi.check(self.lib.wrfgpu_step_launch_count(ctypes.byref(self.params), ctypes.byref(n)))
        self.launches_per_step = int(n.value)

    def alloc_carry(self, like: OperationalCarry) -> OperationalCarry:
        s = like.state
        st = State(**{f_.name: (None if getattr(s, f_.name) is None else torch.empty_like(getattr(s, f_.name)))
                      for f_ in fields(State) if f_.name not in _LEAVES},
                   **{n: getattr(s, n) for n in _LEAVES})
        e = lambda t: torch.empty_like(t)
        return OperationalCarry(state=st, t_2ave=e(s.theta), ww=e(s.w), mudf=e(s.mu_total), muave=e(s.mu_total),
                                muts=e(s.mu_total), ph_tend=e(s.w), u_save=e(s.u), v_save=e(s.v), w_save=e(s.w),
                                t_save=e(s.theta), ph_save=e(s.w), mu_save=e(s.mu_total), ww_save=e(s.w))

    def _structs(self, carry: OperationalCarry, out: OperationalCarry, physics=None):
        """C input/output structs for one step from ``carry`` into ``out``
        (``physics``: a DryPhysicsTendencies-like bundle of device tensors,
        None leaves = zero; only for a stepper built with ``physics=True``)."""
        s, o, nl = carry.state, out.state, self.nl
        if physics is not None and not self.params.physics:
            raise ValueError("physics tendencies given to a stepper built without physics=True")
        ins = _capi.StepInputs()
        if physics is not None:
            for leaf, field in zip(_capi.PHYSICS_LEAVES, _capi.PHYSICS_FIELDS):
                setattr(ins, field, _ptr(getattr(physics, leaf, None)))
        for n in STATE_FIELDS:
            setattr(ins, n, _ptr(getattr(s, n)))
        have_q = s.qv is not None
        for k_, n in enumerate(MOIST):
            ins.q[k_] = _ptr(getattr(s, n)) if have_q else None
        ins.mudf = _ptr(carry.mudf)
        t = nl.tendencies
        ins.base_u, ins.base_v, ins.base_w = _ptr(t.u), _ptr(t.v), _ptr(t.w)
        ins.base_theta, ins.base_mu = _ptr(t.theta), _ptr(t.mu)
        if nl.run_boundary and s.u_bdy is not None:
            ins.u_bdy, ins.v_bdy = _ptr(s.u_bdy), _ptr(s.v_bdy)
            ins.bdy_ntime, _, ins.bdy_width, _, ins.bdy_side_len = s.u_bdy.shape
            if nl.specified_bdy_cadence and s.theta_bdy is not None:
                ins.theta_bdy, ins.ph_bdy, ins.mu_bdy = _ptr(s.theta_bdy), _ptr(s.ph_bdy), _ptr(s.mu_bdy)
            bc = nl.boundary_config
            if not bc.force_geopotential and (bc.nested_ph_relax or bc.nested_ph_spec) and s.ph_bdy is not None:
                ins.ph_bdy = _ptr(s.ph_bdy)
            if not bc.force_geopotential and bc.nested_w_relax and s.w_bdy is not None:
                ins.w_bdy = _ptr(s.w_bdy)
        outs = _capi.StepOutputs()
        for n in STATE_FIELDS:
            setattr(outs, n, _ptr(getattr(o, n)))
        for k_, n in enumerate(MOIST):
            outs.q[k_] = _ptr(getattr(o, n)) if have_q else None
        for n in CARRY_FIELDS:
            setattr(outs, n, _ptr(getattr(out, n)))
        return ins, outs

    def step_into(self, carry: OperationalCarry, out: OperationalCarry, lead_seconds=None, stream=None,
                  physics=None) -> None:
        """Enqueue one step from ``carry`` into the preallocated ``out`` (no sync);
        ``physics`` as in ``rk_scan_step``.  ``lead_seconds``: None, a float,
        or a one-element float64 tensor on the device (the traced-clock form:
        the kernels read it, so no host value is needed)."""
        ins, outs = self._structs(carry, out, physics)
        st = torch.cuda.current_stream(self.device) if stream is None else stream
        ws = self.workspace
        if ws is None:
            with torch.cuda.stream(st):
                ws = torch.empty(self.workspace_bytes, dtype=torch.uint8, device=self.device)
        args = (ctypes.byref(self.params), ctypes.byref(self.metrics), ctypes.byref(ins), ctypes.byref(outs))
        tail = (ctypes.c_void_p(ws.data_ptr()), ctypes.c_size_t(ws.numel()), ctypes.c_void_p(st.cuda_stream))
        if isinstance(lead_seconds, torch.Tensor):
            lead_dev = _device_lead(lead_seconds, self.device)
            rc = self.lib.wrfgpu_rk3_step_device_lead(*args, ctypes.c_void_p(lead_dev.data_ptr()), *tail)
        else:
            lead = float("nan") if lead_seconds is None else float(lead_seconds)
            rc = self.lib.wrfgpu_rk3_step(*args, lead, *tail)
        _capi.check(rc)

    def autotune(self, carry: OperationalCarry, out: OperationalCarry, stream=None) -> tuple[int, int, int]:
        """Pick the kernel tile shapes for this grid by timing candidates
        (overwrites ``out``; synchronises).  Returns (march_levels,
        column_lanes, column_width)."""
        ins, outs = self._structs(carry, out)
        st = torch.cuda.current_stream() if stream is None else stream
        _capi.check(self.lib.wrfgpu_autotune(ctypes.byref(self.params), ctypes.byref(self.metrics),
                                             ctypes.byref(ins), ctypes.byref(outs),
                                             ctypes.c_void_p(self.workspace.data_ptr()),
                                             ctypes.c_size_t(self.workspace.numel()), ctypes.c_void_p(st.cuda_stream)))
        return int(self.params.march_levels), int(self.params.column_lanes), int(self.params.column_width)


class BatchStepper:
    """Several independent domains (ensemble members, nest levels; any sizes)
    advanced together by ``wrfgpu_rk3_step_batched``: one call per step,
    members running concurrently on the library's stream pool."""

    def __init__(self, namelists, device="cuda"):
        self.steppers = [Stepper(nl, device=device) for nl in namelists]
        self.lib = _capi.load()

    def alloc_carries(self, likes):
        return [s.alloc_carry(c) for s, c in zip(self.steppers, likes)]

    def step_into(self, carries, outs, lead_seconds=None, stream=None) -> None:
        n = len(self.steppers)
        if len(carries) != n or len(outs) != n:
            raise ValueError("one carry and one output per member")
        P = (_capi.StepParams * n)(*[s.params for s in self.steppers])
        M = (_capi.Metrics * n)(*[s.metrics for s in self.steppers])
        pairs = [s._structs(c, o) for s, c, o in zip(self.steppers, carries, outs)]
        I = (_capi.StepInputs * n)(*[p[0] for p in pairs])
        O = (_capi.StepOutputs * n)(*[p[1] for p in pairs])
        leads = lead_seconds if isinstance(lead_seconds, (list, tuple)) else [lead_seconds] * n
        L = (ctypes.c_double * n)(*[float("nan") if x is None else float(x) for x in leads])
        W = (ctypes.c_void_p * n)(*[s.workspace.data_ptr() for s in self.steppers])
        B = (ctypes.c_size_t * n)(*[s.workspace.numel() for s in self.steppers])
        st = torch.cuda.current_stream() if stream is None else stream
        _capi.check(self.lib.wrfgpu_rk3_step_batched(n, P, M, I, O, L, W, B, ctypes.c_void_p(st.cuda_stream)))


def _same_device(a, b) -> bool:
    a, b = torch.device(a), torch.device(b)
    if a.type != b.type:
        return False
    cur = torch.cuda.current_device() if a.type == "cuda" else 0
    return (cur if a.index is None else a.index) == (cur if b.index is None else b.index)


def _device_lead(t: torch.Tensor, device) -> torch.Tensor:
    if t.numel() != 1 or t.dtype != torch.float64 or not _same_device(t.device, device):
        raise ValueError("a device lead_seconds must be one float64 element on the step's device")
    return t.reshape(1)


# Prepared steps (params and metric pointers, no workspace) of recent
# namelists, keyed by their content so that a caller who builds a new
# namelist per call (the reference's ``namelist.replace(...)`` idiom) reuses
# them; bounded, least recently used evicted first.
_PLANS: "OrderedDict[tuple, Stepper]" = OrderedDict()
_PLAN_CAPACITY = 8


def _plan_key(nl: OperationalNamelist, physics: bool, device) -> tuple:
    p = step_params(nl)
    m = nl.metrics
    ptrs = tuple(getattr(m, n).data_ptr() for n in METRIC_ARRAYS)
    return bytes(ctypes.string_at(ctypes.addressof(p), ctypes.sizeof(p))), ptrs, bool(physics), str(device)


def _plan_for(nl: OperationalNamelist, physics: bool, device) -> Stepper:
    key = _plan_key(nl, physics, device)
    stp = _PLANS.get(key)
    if stp is None:
        stp = Stepper(nl, device=device, physics=physics, own_workspace=False)
        _PLANS[key] = stp
        while len(_PLANS) > _PLAN_CAPACITY:
            _PLANS.popitem(last=False)
    else:
        _PLANS.move_to_end(key)
        stp.nl = nl  # the base tendencies are read from the namelist at call time
    return stp


@dataclass
class PreHaloCaptureResult:
    """``_PreHaloCaptureResult`` (operational_mode.py): carry + pre-halo state.
    On one GPU the halo exchange is a no-op, so both are the same state."""

    carry: OperationalCarry
    pre_halo_state: State


def rk_scan_step(carry: OperationalCarry, namelist: OperationalNamelist, *, debug: bool = False, lead_seconds=None,
                 physics_tendencies=None, capture_pre_halo: bool = False):
    """Drop-in for ``_rk_scan_step`` (runtime/operational_mode.py:3319-3534).

    Returns a new ``OperationalCarry``; ``carry`` is not modified.  The step is
    enqueued on the current CUDA stream and is not synchronised; its scratch
    comes from torch's caching allocator on that stream, so calls on
    different streams never share a workspace.  ``lead_seconds`` is None, a
    float, or a one-element float64 device tensor (the reference's traced
    clock: the kernels read it, so the call can sit in a captured graph whose
    replays advance the clock on the device).
    ``physics_tendencies`` is a DryPhysicsTendencies-like bundle
    (dynamics/core/rk_addtend_dry.py:103-124: ru_tendf, rv_tendf, rw_tendf,
    ph_tendf, t_tendf, mu_tendf, h_diabatic, u_save, v_save, w_save, ph_save,
    t_save; float64 CUDA tensors, absent or None leaves are zero) merged into
    every RK stage as rk_addtend_dry does.
    """
    reason = _unsupported(namelist, physics_tendencies)
    if reason:
        raise NotImplementedError(reason)
    with_physics = physics_tendencies is not None
    stp = _plan_for(namelist, with_physics, carry.state.u.device)
    if carry.mudf is None:
        carry = carry.replace(mudf=torch.zeros_like(carry.state.mu_total))
    out = stp.alloc_carry(carry)
    stp.step_into(carry, out, lead_seconds=lead_seconds, physics=physics_tendencies)
    out.base_state = carry.base_state
    if debug:
        print("wrfgpu rk3 step: 3 stages, substeps", 1, max(1, namelist.acoustic_substeps // 2),
              namelist.acoustic_substeps)
    if capture_pre_halo:
        return PreHaloCaptureResult(out, out.state)
    return out


def carry_from_case(case, device="cuda") -> OperationalCarry:
    st = State.from_host(case.state, device)
    c = initial_operational_carry(st)
    return c.replace(mudf=_dev(case.mudf, device))


def _state_structs(state: State):
    """The state's leaves as a wrfgpu_step_inputs, and a fresh State (the
    strips carried over) with its wrfgpu_step_outputs."""
    out = State(**{f_.name: (torch.empty_like(getattr(state, f_.name)) if getattr(state, f_.name) is not None
                             and f_.name not in _LEAVES else getattr(state, f_.name)) for f_ in fields(State)})
    outs = _capi.StepOutputs()
    for n in STATE_FIELDS:
        setattr(outs, n, _ptr(getattr(out, n)))
    for k_, n in enumerate(MOIST):
        outs.q[k_] = _ptr(getattr(out, n))
    return _inputs_struct(state), out, outs


def _inputs_struct(state: State) -> _capi.StepInputs:
    ins = _capi.StepInputs()
    for n in STATE_FIELDS:
        setattr(ins, n, _ptr(getattr(state, n)))
    for k_, n in enumerate(MOIST):
        ins.q[k_] = _ptr(getattr(state, n))
    return ins


def _leaves_struct(state: State) -> _capi.LbcLeaves:
    nz = state.theta.shape[0]
    lv = _capi.LbcLeaves()
    lv.u, lv.v, lv.w, lv.theta = _ptr(state.u_bdy), _ptr(state.v_bdy), _ptr(state.w_bdy), _ptr(state.theta_bdy)
    for k_, n in enumerate(MOIST):
        lv.q[k_] = _ptr(getattr(state, n + "_bdy"))
    lv.p, lv.pb, lv.mu, lv.mub = _ptr(state.p_bdy), _ptr(state.pb_bdy), _ptr(state.mu_bdy), _ptr(state.mub_bdy)
    lv.ph, lv.phb = _ptr(state.ph_bdy), _ptr(state.phb_bdy)
    lv.ntime, _, lv.width, _, lv.side_len = state.u_bdy.shape
    levels = dict(w_bdy=nz + 1, ph_bdy=nz + 1, phb_bdy=nz + 1, mu_bdy=1, mub_bdy=1)
    for n in _LEAVES:
        t = getattr(state, n)
        if t is not None and tuple(t.shape) != (lv.ntime, 4, lv.width, levels.get(n, nz), lv.side_len):
            raise ValueError(f"{n} has shape {tuple(t.shape)}, expected "
                             f"{(lv.ntime, 4, lv.width, levels.get(n, nz), lv.side_len)}")
    return lv


def apply_lateral_boundaries(state: State, lead_seconds, dt_s: float, config: BoundaryConfig | None = None,
                             metrics=None, *, dry_spec_only: bool = False) -> State:
    """Drop-in for ``apply_lateral_boundaries`` (coupling/boundary_apply.py:170-326),
    the forecast step's end-of-step lateral boundary pass, through
    ``wrfgpu_apply_lateral_boundaries``: the state's ``*_bdy`` strips at
    ``lead_seconds`` relax the boundary band and set the outer row (or, with
    ``dry_spec_only``, set the outer row only).  Returns a new State (the
    strips carried over); enqueued on the current stream, not synchronised.
    ``metrics`` is accepted for the reference's signature and not needed."""
    del metrics
    cfg = BoundaryConfig() if config is None else config
    lib = _capi.load()
    nz, ny, nx = state.theta.shape
    p = _capi.StepParams()
    lib.wrfgpu_step_params_init(ctypes.byref(p))
    p.nx, p.ny, p.nz, p.dx, p.dy, p.dt = nx, ny, nz, 1.0, 1.0, float(dt_s)
    p.spec_zone, p.relax_zone = int(cfg.spec_zone), int(cfg.relax_zone)
    p.update_cadence_s = float(cfg.update_cadence_s)
    p.force_geopotential = int(bool(cfg.force_geopotential))
    ins, out, outs = _state_structs(state)
    lv = _leaves_struct(state)
    st = torch.cuda.current_stream(state.u.device)
    _capi.check(lib.wrfgpu_apply_lateral_boundaries(ctypes.byref(p), ctypes.byref(ins), ctypes.byref(lv),
                                                     ctypes.byref(outs), float(lead_seconds),
                                                     int(bool(dry_spec_only)), ctypes.c_void_p(st.cuda_stream)))
    return out


def theta_limiter_diagnostics(raw: torch.Tensor) -> dict:
    """The limiter record (``wrfgpu_theta_limiter_diag``, 40 bytes on the
    device) as the reference's dict of device scalars
    (operational_mode.py:1444-1454)."""
    ints, dbl = raw[:16].view(torch.int32), raw[16:].view(torch.float64)
    return {"theta_limited_cell_count": ints[0], "theta_first_limited_cell_xyz": ints[1:4],
            "theta_mass_before": dbl[0], "theta_mass_after": dbl[1], "theta_mass_residual": dbl[2]}


def step_epilogue(next_state: State, origin: State, lead_seconds, nl: OperationalNamelist):
    """The forecast step after ``_rk_scan_step`` without physics
    (runtime/operational_mode.py:4950-4983), through ``wrfgpu_step_epilogue``:
    unless ``nl.disable_guards``, the theta increment limiter, dry-mass and
    mixing-ratio guards against ``origin`` (the step-start state); with
    ``nl.run_boundary`` the end-of-step lateral boundary pass (ring 0 only
    when the specified boundary cadence is active) and the guards of the
    bounded state.  ``lead_seconds`` is a float or a one-element float64
    device tensor (read by the boundary kernels).  Returns (State, limiter
    diagnostics); enqueued on the current stream, not synchronised."""
    lib = _capi.load()
    p = step_params(nl)
    dev = next_state.u.device
    n = ctypes.c_size_t(0)
    _capi.check(lib.wrfgpu_step_epilogue_workspace_size(ctypes.byref(p), ctypes.byref(n)))
    ws = torch.empty(n.value + 256, dtype=torch.uint8, device=dev)
    wsp = (ws.data_ptr() + 255) // 256 * 256
    raw = torch.empty(_capi.THETA_DIAG_BYTES, dtype=torch.uint8, device=dev)
    ins, out, outs = _state_structs(next_state)
    org = _inputs_struct(origin)
    lv = _leaves_struct(next_state) if nl.run_boundary else None
    st = torch.cuda.current_stream(dev)
    head = (ctypes.byref(p), ctypes.byref(org), ctypes.byref(ins), None if lv is None else ctypes.byref(lv),
            ctypes.byref(outs))
    tail = (int(bool(nl.disable_guards)), ctypes.c_void_p(raw.data_ptr()), ctypes.c_void_p(wsp), n.value,
            ctypes.c_void_p(st.cuda_stream))
    if isinstance(lead_seconds, torch.Tensor):
        lead_dev = _device_lead(lead_seconds, dev)
        _capi.check(lib.wrfgpu_step_epilogue_device_lead(*head, ctypes.c_void_p(lead_dev.data_ptr()), *tail))
    else:
        _capi.check(lib.wrfgpu_step_epilogue(*head, float(lead_seconds), *tail))
    return out, theta_limiter_diagnostics(raw)


def forecast_step(carry: OperationalCarry, namelist: OperationalNamelist, step_index, *, debug: bool = False):
    """One forecast step without physics, as the reference's
    ``_physics_boundary_step_with_limiter_diagnostics``
    (runtime/operational_mode.py:4915-4993) runs it with physics off: the
    clock ``lead_seconds = step_index * dt``, ``rk_scan_step`` at that lead,
    then the post-step guards and the end-of-step lateral boundary pass
    (``step_epilogue``; ring 0 only under the specified boundary cadence).
    ``step_index`` is an int or a one-element float64 device tensor (then the
    lead is formed on the device and the step reads it there).  Returns the
    new carry and the theta limiter's diagnostics; not synchronised."""
    if isinstance(step_index, torch.Tensor):
        lead = (step_index.to(torch.float64) * float(namelist.dt_s)).reshape(1)
    else:
        lead = float(step_index) * float(namelist.dt_s)
    origin = carry.state
    nxt = rk_scan_step(carry, namelist, debug=debug, lead_seconds=lead)
    state, diag = step_epilogue(nxt.state, origin, lead, namelist)
    return nxt.replace(state=state), diag
