"""Nest coupling around the step, on the CUDA C ABI.

A nested child domain is forced at its lateral boundary by its parent and may
feed its interior back onto the parent.  This module mirrors the reference's
host API for both directions:

* ``build_nest_force_weights`` (src/gpuwrf/nesting/boundary_construction.py:
  117-146) builds the static parent -> child gathers of the mass, u and v
  staggerings (nesting/interp.py:109-245: WRF ``sint`` cell-centered
  registration ``x = (start - 1) + (i - ratio // 2) / ratio`` by default, or
  the node-aligned one; coordinates clipped into the parent, floor / ceil
  corner indices and the toward-ceil weight);
* ``build_child_boundary_package`` (boundary_construction.py:360-451) fills the
  child's eleven ``*_bdy`` leaves with the two-time package [the child's own
  ring, the parent interpolated to it] (``wrfgpu_nest_ring_leaf``);
* ``interp_parent_field_to_child`` (:454-468) interpolates a whole field
  (``wrfgpu_nest_interp_field``);
* ``build_state_feedback_weights`` (coupling/boundary_feedback.py:170-357)
  builds the WRF ``copy_fcn`` odd-ratio feedback plans and the ``sm121``
  smoother interiors;
* ``apply_state_feedback`` (:509-592) writes the child's overlap means onto
  the parent, smooths the overlap and rebuilds the totals
  (``wrfgpu_nest_feedback``, ``wrfgpu_nest_rebuild_total``).

The plans are built once on the host from the static nest geometry (as the
reference builds them); every per-call operation runs in ``libwrfgpu.so`` on
the current CUDA stream.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, replace

import numpy as np
import torch

from . import _capi
from .dycore import State, _ptr

FORCED_LEAVES = ("u_bdy", "v_bdy", "w_bdy", "theta_bdy", "qv_bdy", "ph_bdy", "phb_bdy", "p_bdy", "pb_bdy", "mu_bdy",
                 "mub_bdy")


@dataclass
class InterpWeights:
    """Static parent -> child gather of one staggering (device arrays)."""

    y0: torch.Tensor
    y1: torch.Tensor
    x0: torch.Tensor
    x1: torch.Tensor
    wy: torch.Tensor
    wx: torch.Tensor
    child_ny: int
    child_nx: int
    parent_ny: int
    parent_nx: int

    def c_struct(self) -> _capi.NestInterp:
        return _capi.NestInterp(_ptr_int(self.y0), _ptr_int(self.y1), _ptr_int(self.x0), _ptr_int(self.x1),
                                _ptr(self.wy), _ptr(self.wx), self.child_ny, self.child_nx, self.parent_ny,
                                self.parent_nx)


@dataclass
class NestForceWeights:
    mass: InterpWeights
    u: InterpWeights
    v: InterpWeights
    registration: str


def _ptr_int(t: torch.Tensor) -> int:
    if t.dtype != torch.int32 or not t.is_contiguous() or not t.is_cuda:
        raise ValueError("index arrays must be contiguous int32 CUDA tensors")
    return t.data_ptr()


def _axis(start_1based: int, child_len: int, ratio: int, parent_len: int, cell_centered: bool):
    idx = np.arange(int(child_len), dtype=np.float64)
    base = float(int(start_1based) - 1)
    coords = base + ((idx - float(int(ratio) // 2)) / float(ratio) if cell_centered else idx / float(ratio))
    c = np.clip(coords, 0.0, float(parent_len - 1))
    lo = np.floor(c).astype(np.int64)
    hi = np.clip(lo + 1, 0, parent_len - 1)
    return lo.astype(np.int32), hi.astype(np.int32), c - lo.astype(np.float64)


def _weights(ratio, i_start, j_start, pny, pnx, cny, cnx, registration, device) -> InterpWeights:
    if int(ratio) <= 1:
        raise ValueError(f"nested child requires parent_grid_ratio > 1, got {ratio}")
    cc = registration == "sint"
    y0, y1, wy = _axis(j_start, cny, ratio, pny, cc)
    x0, x1, wx = _axis(i_start, cnx, ratio, pnx, cc)
    t = lambda a: torch.as_tensor(a, device=device)
    return InterpWeights(t(y0), t(y1), t(x0), t(x1), t(wy), t(wx), int(cny), int(cnx), int(pny), int(pnx))


def build_nest_force_weights(*, parent_grid_ratio: int, i_parent_start: int, j_parent_start: int, parent_grid,
                             child_grid, registration: str = "sint", device="cuda") -> NestForceWeights:
    """Mass / u / v parent -> child gathers of one nest edge
    (boundary_construction.py:117-146).  ``parent_grid`` / ``child_grid`` are
    anything with ``nx`` and ``ny`` (mass-grid extents)."""
    if registration not in ("sint", "bilinear"):
        raise ValueError(f"unknown nest interpolation registration {registration!r}")
    pny, pnx, cny, cnx = int(parent_grid.ny), int(parent_grid.nx), int(child_grid.ny), int(child_grid.nx)
    c = (parent_grid_ratio, i_parent_start, j_parent_start)
    return NestForceWeights(mass=_weights(*c, pny, pnx, cny, cnx, registration, device),
                            u=_weights(*c, pny, pnx + 1, cny, cnx + 1, registration, device),
                            v=_weights(*c, pny + 1, pnx, cny + 1, cnx, registration, device),
                            registration=registration)


def interp_parent_field_to_child(field: torch.Tensor, weights: NestForceWeights, *,
                                 staggering: str = "mass") -> torch.Tensor:
    """A parent field interpolated onto the whole child grid (2-D or 3-D)."""
    w = {"mass": weights.mass, "u": weights.u, "v": weights.v}[staggering]
    f3 = field if field.dim() == 3 else field.unsqueeze(0)
    if tuple(f3.shape[1:]) != (w.parent_ny, w.parent_nx):
        raise ValueError(f"field {tuple(field.shape)} does not match the parent extent {(w.parent_ny, w.parent_nx)}")
    out = torch.empty((f3.shape[0], w.child_ny, w.child_nx), dtype=torch.float64, device=field.device)
    st = torch.cuda.current_stream(field.device)
    lib = _capi.load()
    _capi.check(lib.wrfgpu_nest_interp_field(ctypes.byref(w.c_struct()), _ptr(f3.contiguous()), int(f3.shape[0]),
                                             _ptr(out), ctypes.c_void_p(st.cuda_stream)))
    return out if field.dim() == 3 else out[0]


def build_child_boundary_package(child_state: State, parent_state: State, weights: NestForceWeights, *,
                                 bdy_width: int = 5) -> State:
    """The child's two-time boundary package from its parent
    (boundary_construction.py:360-451): u, v, w, theta, qv, ph', p', mu' from
    the parent at time 1; phb, pb, mub from the child's own base at both
    times.  Returns a new State (the interior untouched)."""
    if int(bdy_width) <= 0:
        raise ValueError(f"bdy_width must be positive, got {bdy_width}")
    w = int(bdy_width)
    side_len = int(max(child_state.u_bdy.shape[-1], child_state.v_bdy.shape[-1]))
    lib = _capi.load()
    st = torch.cuda.current_stream(child_state.u.device)
    cs = child_state
    jobs = {  # leaf: (child field, subtracted child field or None, parent field or None, weights)
        "u_bdy": (cs.u, None, parent_state.u, weights.u),
        "v_bdy": (cs.v, None, parent_state.v, weights.v),
        "w_bdy": (cs.w, None, parent_state.w, weights.mass),
        "theta_bdy": (cs.theta, None, parent_state.theta, weights.mass),
        "qv_bdy": (cs.qv, None, parent_state.qv, weights.mass),
        "ph_bdy": (cs.ph_perturbation, None, parent_state.ph_perturbation, weights.mass),
        "phb_bdy": (cs.ph_total, cs.ph_perturbation, None, None),  # the child's own base
        "p_bdy": (cs.p_perturbation, None, parent_state.p_perturbation, weights.mass),
        "pb_bdy": (cs.p_total, cs.p_perturbation, None, None),
        "mu_bdy": (cs.mu_perturbation, None, parent_state.mu_perturbation, weights.mass),
        "mub_bdy": (cs.mu_total, cs.mu_perturbation, None, None),
    }
    new = {}
    for name, (cf, csub, pf, wt) in jobs.items():
        old = getattr(child_state, name)
        if old is None:
            raise ValueError(f"the child state has no {name} leaf to fit the package to")
        lz, lside = int(old.shape[-2]), int(old.shape[-1])
        c3 = (cf if cf.dim() == 3 else cf.unsqueeze(0)).contiguous()
        s3 = None if csub is None else (csub if csub.dim() == 3 else csub.unsqueeze(0)).contiguous()
        leaf = torch.empty((2, 4, w, lz, lside), dtype=torch.float64, device=cf.device)
        if pf is not None:
            p3 = (pf if pf.dim() == 3 else pf.unsqueeze(0)).contiguous()
            wp = ctypes.byref(wt.c_struct())
        else:
            p3, wp = None, None
        _capi.check(lib.wrfgpu_nest_ring_leaf(wp, None if p3 is None else _ptr(p3), _ptr(c3),
                                              None if s3 is None else _ptr(s3), int(c3.shape[0]),
                                              int(c3.shape[1]), int(c3.shape[2]), w, side_len, lz, lside,
                                              _ptr(leaf), ctypes.c_void_p(st.cuda_stream)))
        new[name] = leaf
    return replace(child_state, **new)


@dataclass
class FeedbackPlan:
    parent_lin: torch.Tensor
    child_lin: torch.Tensor
    pwe: int
    psn: int
    cwe: int
    csn: int
    stencil: int
    i_lo: int
    i_hi: int
    j_lo: int
    j_hi: int

    def c_struct(self, smooth: bool) -> _capi.NestFeedbackPlan:
        n = int(self.parent_lin.numel())
        return _capi.NestFeedbackPlan(_ptr_int(self.parent_lin) if n else None,
                                      _ptr_int(self.child_lin) if n else None, n, self.stencil, self.pwe, self.psn,
                                      self.cwe, self.csn, self.i_lo, self.i_hi, self.j_lo, self.j_hi, int(smooth))


@dataclass
class StateFeedbackWeights:
    mass: FeedbackPlan
    u: FeedbackPlan
    v: FeedbackPlan
    smooth_option: int = 1


def _feedback_plan(ratio, ipos, jpos, pwe0, psn0, cwe0, csn0, stagger, spec_zone, device) -> FeedbackPlan:
    """WRF copy_fcn odd-ratio donors (boundary_feedback.py:170-267) and the
    sm121 interior (:270-319) of one staggering."""
    r = int(ratio)
    if r <= 1:
        raise ValueError(f"feedback requires parent_grid_ratio > 1, got {r}")
    if r % 2 == 0:
        raise NotImplementedError("feedback supports the WRF odd-ratio copy_fcn branch")
    pwe, psn = pwe0 + (stagger == "U"), psn0 + (stagger == "V")
    cwe, csn = cwe0 + (stagger == "U"), csn0 + (stagger == "V")
    istag, jstag = (0 if stagger == "U" else 1), (0 if stagger == "V" else 1)
    n_pi, n_pj, h = cwe0 // r, csn0 // r, r // 2
    cj = np.arange(jpos + spec_zone, jpos + n_pj - jstag - spec_zone + 1)
    ci = np.arange(ipos + spec_zone, ipos + n_pi - istag - spec_zone + 1)
    CJ, CI = np.meshgrid(cj, ci, indexing="ij")
    CJ, CI = CJ.ravel(), CI.ravel()
    if stagger == "":
        ni, nj = (CI - ipos) * r + h + 1, (CJ - jpos) * r + h + 1
        jj, ii = np.meshgrid(np.arange(r) - h, np.arange(r) - h, indexing="ij")
        rows = nj[:, None] + jj.ravel()[None, :] - 1
        cols = ni[:, None] + ii.ravel()[None, :] - 1
    elif stagger == "U":
        ni, nj = (CI - ipos) * r + 1, (CJ - jpos) * r + h + 1
        rows = nj[:, None] + (np.arange(r) - h)[None, :] - 1
        cols = np.repeat((ni - 1)[:, None], r, axis=1)
    else:
        ni, nj = (CI - ipos) * r + h + 1, (CJ - jpos) * r + 1
        rows = np.repeat((nj - 1)[:, None], r, axis=1)
        cols = ni[:, None] + (np.arange(r) - h)[None, :] - 1
    if rows.size and (rows.min() < 0 or rows.max() >= csn or cols.min() < 0 or cols.max() >= cwe):
        raise IndexError(f"feedback donor out of bounds of the child extent ({csn}, {cwe})")
    child_lin = (rows * cwe + cols).astype(np.int32).reshape(-1, r * r if stagger == "" else r)
    parent_lin = ((CJ - 1) * pwe + (CI - 1)).astype(np.int32)
    i_lo1, i_hi1 = ipos + 2, ipos + n_pi - 2 - istag
    j_lo1, j_hi1 = jpos + 2, jpos + n_pj - 2 - jstag
    i_lo, i_hi = max(i_lo1 - 1, 0), max(i_hi1, i_lo1 - 1)
    j_lo, j_hi = max(j_lo1 - 1, 0), max(j_hi1, j_lo1 - 1)
    # the smoother never reads outside the parent field (boundary_feedback.py:459-474)
    if i_lo < 1 or i_hi > pwe - 1 or j_lo < 1 or j_hi > psn - 1:
        i_lo, i_hi, j_lo, j_hi = max(i_lo, 1), min(i_hi, pwe - 1), max(j_lo, 1), min(j_hi, psn - 1)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=device)
    return FeedbackPlan(t(parent_lin), t(child_lin), int(pwe), int(psn), int(cwe), int(csn), child_lin.shape[1],
                        int(i_lo), int(i_hi), int(j_lo), int(j_hi))


def build_state_feedback_weights(*, parent_grid_ratio: int, i_parent_start: int, j_parent_start: int, parent_grid,
                                 child_grid, spec_zone: int = 1, smooth_option: int = 1,
                                 device="cuda") -> StateFeedbackWeights:
    """Mass / U / V feedback plans with their sm121 interiors for one edge
    (boundary_feedback.py:322-357)."""
    c = (parent_grid_ratio, int(i_parent_start), int(j_parent_start), int(parent_grid.nx), int(parent_grid.ny),
         int(child_grid.nx), int(child_grid.ny))
    return StateFeedbackWeights(mass=_feedback_plan(*c, "", int(spec_zone), device),
                                u=_feedback_plan(*c, "U", int(spec_zone), device),
                                v=_feedback_plan(*c, "V", int(spec_zone), device),
                                smooth_option=int(smooth_option))


def _feedback_field(parent: torch.Tensor, child: torch.Tensor, plan: FeedbackPlan, smooth: bool) -> torch.Tensor:
    p3 = (parent if parent.dim() == 3 else parent.unsqueeze(0)).contiguous()
    c3 = (child if child.dim() == 3 else child.unsqueeze(0)).contiguous()
    if tuple(p3.shape[1:]) != (plan.psn, plan.pwe) or tuple(c3.shape[1:]) != (plan.csn, plan.cwe):
        raise ValueError("feedback field shapes do not match the plan")
    if p3.shape[0] != c3.shape[0]:
        raise ValueError("parent and child fields have different level counts")
    out = torch.empty_like(p3)
    scratch = torch.empty_like(p3) if smooth else None
    st = torch.cuda.current_stream(parent.device)
    lib = _capi.load()
    _capi.check(lib.wrfgpu_nest_feedback(ctypes.byref(plan.c_struct(smooth)), _ptr(p3), _ptr(c3), int(p3.shape[0]),
                                         _ptr(out), None if scratch is None else _ptr(scratch),
                                         ctypes.c_void_p(st.cuda_stream)))
    return out if parent.dim() == 3 else out[0]


def _rebuild_total(parent_total, parent_pert, new_pert) -> torch.Tensor:
    out = torch.empty_like(new_pert)
    st = torch.cuda.current_stream(new_pert.device)
    lib = _capi.load()
    _capi.check(lib.wrfgpu_nest_rebuild_total(_ptr(parent_total.contiguous()), _ptr(parent_pert.contiguous()),
                                              _ptr(new_pert), new_pert.numel(), _ptr(out),
                                              ctypes.c_void_p(st.cuda_stream)))
    return out


def apply_state_feedback(parent: State, child: State, weights: StateFeedbackWeights, *,
                         feedback: bool = True) -> State:
    """Two-way feedback onto the parent (boundary_feedback.py:509-592): the
    overlap means of u, v (their own plans), w, theta, qv, p', ph', mu' and
    the carried species (mass plan), each smoothed by sm121 unless
    ``smooth_option`` is 0; the parent's base kept and the totals rebuilt.
    Returns a new State; ``feedback=False`` returns ``parent`` itself."""
    if not feedback:
        return parent
    sm = weights.smooth_option != 0
    fb = lambda p, c, plan: _feedback_field(p, c, plan, sm)
    up = dict(u=fb(parent.u, child.u, weights.u), v=fb(parent.v, child.v, weights.v),
              w=fb(parent.w, child.w, weights.mass), theta=fb(parent.theta, child.theta, weights.mass),
              qv=fb(parent.qv, child.qv, weights.mass),
              p_perturbation=fb(parent.p_perturbation, child.p_perturbation, weights.mass),
              ph_perturbation=fb(parent.ph_perturbation, child.ph_perturbation, weights.mass),
              mu_perturbation=fb(parent.mu_perturbation, child.mu_perturbation, weights.mass))
    up["p_total"] = _rebuild_total(parent.p_total, parent.p_perturbation, up["p_perturbation"])
    up["ph_total"] = _rebuild_total(parent.ph_total, parent.ph_perturbation, up["ph_perturbation"])
    up["mu_total"] = _rebuild_total(parent.mu_total, parent.mu_perturbation, up["mu_perturbation"])
    for q in ("qc", "qr", "qi", "qs", "qg"):
        pv, cv = getattr(parent, q), getattr(child, q)
        if pv is not None and cv is not None:
            up[q] = fb(pv, cv, weights.mass)
    return replace(parent, **up)


# ---------------------------------------------------------------------------
# The nest tower: WRF's integrate recursion on the device
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class NestEdge:
    """Static parent -> child geometry of one tower edge
    (nesting/scheduler.py:49-62): the space / time ratio and the 1-based
    origin of the child in the parent grid."""

    parent: str
    child: str
    parent_grid_ratio: int
    i_parent_start: int
    j_parent_start: int


class NestTower:
    """A nested tower advanced the way WRF's ``integrate`` recursion does
    (frame/module_integrate.F:408-435 as nesting/scheduler.py:191-224
    restates it): per own step of a domain, (1) advance it one forecast step
    (``dycore.forecast_step``: RK3 step, guards, end-of-step boundary pass),
    (2) build every child's two-time boundary package from the just-advanced
    domain, (3) recurse into each child for ``parent_grid_ratio`` own steps,
    (4) with ``feedback`` write the child back onto the parent
    (``apply_state_feedback``).  Every domain's forecast clock inside its
    parent's step is ``local_step * dt`` (local_step 1-based), so a child's
    strips (update cadence = its parent's dt) are interpolated from the old
    ring at 0 to the parent's new state at the parent's step end.

    ``namelists[name]``: each domain's namelist; a child must be a nested
    boundary domain (run_boundary, non-ideal source, force_geopotential off)
    with dt = parent dt / ratio and update_cadence_s = parent dt.
    ``grids[name]``: mass-grid extents (``nx``, ``ny``)."""

    def __init__(self, order, edges, namelists, grids, *, registration: str = "sint", feedback: bool = False,
                 bdy_width: int = 5, smooth_option: int = 1, device="cuda"):
        self.order = list(order)
        self.edges: dict[str, list[NestEdge]] = {}
        for e in edges:
            self.edges.setdefault(e.parent, []).append(e)
        self.namelists = dict(namelists)
        self.feedback = bool(feedback)
        self.bdy_width = int(bdy_width)
        self.force_w, self.fb_w = {}, {}
        for e in edges:
            pn, cn = self.namelists[e.parent], self.namelists[e.child]
            r = int(e.parent_grid_ratio)
            bc = cn.boundary_config
            if not (cn.run_boundary and cn.bc_source != "ideal" and not bc.force_geopotential):
                raise ValueError(f"{e.child}: a nest child must be a nested boundary domain "
                                 "(run_boundary, non-ideal bc_source, force_geopotential off)")
            if abs(cn.dt_s * r - pn.dt_s) > 1e-9 * pn.dt_s:
                raise ValueError(f"{e.child}: dt_s must be the parent's dt_s / parent_grid_ratio")
            if abs(bc.update_cadence_s - pn.dt_s) > 1e-9 * pn.dt_s:
                raise ValueError(f"{e.child}: update_cadence_s must be the parent's dt_s")
            c = dict(parent_grid_ratio=r, i_parent_start=e.i_parent_start, j_parent_start=e.j_parent_start,
                     parent_grid=grids[e.parent], child_grid=grids[e.child])
            self.force_w[e.child] = build_nest_force_weights(registration=registration, device=device, **c)
            if self.feedback:
                self.fb_w[e.child] = build_state_feedback_weights(smooth_option=smooth_option, device=device, **c)

    def run(self, carries: dict, root_steps: int, root: str | None = None) -> dict:
        """Advance the tower ``root_steps`` steps of its root; returns the new
        carries (``carries`` itself is not modified)."""
        from .dycore import forecast_step

        out = dict(carries)
        root = root or self.order[0]

        def integrate(name: str, n_steps: int) -> None:
            children = self.edges.get(name, [])
            for local in range(1, int(n_steps) + 1):
                out[name], _ = forecast_step(out[name], self.namelists[name], local)
                for e in children:
                    pkg = build_child_boundary_package(out[e.child].state, out[name].state, self.force_w[e.child],
                                                       bdy_width=self.bdy_width)
                    out[e.child] = out[e.child].replace(state=pkg)
                for e in children:
                    integrate(e.child, int(e.parent_grid_ratio))
                    if self.feedback:
                        fed = apply_state_feedback(out[name].state, out[e.child].state, self.fb_w[e.child])
                        out[name] = out[name].replace(state=fed)

        integrate(root, int(root_steps))
        return out
