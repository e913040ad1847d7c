"""CPU oracle (test infrastructure only) of the nest coupling around the step.

NumPy float64 restatement of the reference's parent->child boundary
construction and child->parent feedback:

* ``src/gpuwrf/nesting/interp.py``: static bilinear gather weights with the
  node-aligned (``:127-150`` cell_centered=False) or WRF cell-centered
  ``sint`` registration (``x = (start-1) + (i - ratio//2)/ratio``), clipped
  floor / ceil indices and the toward-ceil weight (``:109-124``), and the
  y-then-x gather (``:248-277``);
* ``src/gpuwrf/nesting/boundary_construction.py``: the ring strips
  (``field_sides_3d/_2d``, ``:162-210``; W, E flipped, S, N flipped, zero
  padded), the leaf fit (``:347-357``) and the two-time child boundary package
  (``build_child_boundary_package``, ``:360-451``: time 0 the child's own ring,
  time 1 the parent interpolated to it; the base leaves from the child's own
  base at both times);
* ``src/gpuwrf/coupling/boundary_feedback.py``: WRF ``copy_fcn`` odd-ratio
  feedback plans (``:170-267``), the overlap mean written onto the parent
  (``:362-425``), the ``sm121`` 1-2-1 smoother of the overlap interior
  (``:270-319, 428-494``) and the state feedback with totals rebuilt from the
  parent base (``:509-592``).

Only the tests, ``smoke()`` and bench's CPU baseline import it.  The
stencil means are summed in donor order (the GPU kernels sum the same way);
the reference's XLA reduction order is not specified, so the two may differ
from the reference in the last ulp of a mean.
"""

from __future__ import annotations

from dataclasses import dataclass
from types import SimpleNamespace

import numpy as np


# ---------------------------------------------------------------------------
# parent -> child interpolation weights and gather
# ---------------------------------------------------------------------------

@dataclass
class InterpWeights:
    y0: np.ndarray
    y1: np.ndarray
    x0: np.ndarray
    x1: np.ndarray
    wy: np.ndarray
    wx: np.ndarray
    child_ny: int
    child_nx: int


def _axis_weights(coords, parent_size):
    clamped = np.clip(np.asarray(coords, dtype=np.float64), 0.0, float(parent_size - 1))
    lower = np.floor(clamped).astype(np.int64)
    upper = np.clip(lower + 1, 0, parent_size - 1)
    return lower.astype(np.int32), upper.astype(np.int32), clamped - lower.astype(np.float64)


def _axis_coords(start_1based, child_len, ratio, cell_centered):
    base = float(int(start_1based) - 1)
    idx = np.arange(int(child_len), dtype=np.float64)
    if cell_centered:
        return base + (idx - float(int(ratio) // 2)) / float(ratio)
    return base + idx / float(ratio)


def build_interp_weights(*, ratio, i_parent_start, j_parent_start, parent_ny, parent_nx, child_ny, child_nx,
                         registration="sint"):
    if registration not in ("sint", "bilinear"):
        raise ValueError(registration)
    if int(ratio) <= 1:
        raise ValueError("nested child requires parent_grid_ratio > 1")
    cc = registration == "sint"
    y0, y1, wy = _axis_weights(_axis_coords(j_parent_start, child_ny, ratio, cc), parent_ny)
    x0, x1, wx = _axis_weights(_axis_coords(i_parent_start, child_nx, ratio, cc), parent_nx)
    return InterpWeights(y0, y1, x0, x1, wy, wx, int(child_ny), int(child_nx))


def interp(field, w: InterpWeights):
    """y first, then x, as interp.py:248-277."""
    if field.ndim == 2:
        return interp(field[None], w)[0]
    f_y = (1.0 - w.wy[None, :, None]) * field[:, w.y0, :] + w.wy[None, :, None] * field[:, w.y1, :]
    return (1.0 - w.wx[None, None, :]) * f_y[:, :, w.x0] + w.wx[None, None, :] * f_y[:, :, w.x1]


def build_nest_force_weights(*, ratio, i_parent_start, j_parent_start, parent_ny, parent_nx, child_ny, child_nx,
                             registration="sint"):
    c = dict(ratio=ratio, i_parent_start=i_parent_start, j_parent_start=j_parent_start, registration=registration)
    return SimpleNamespace(
        mass=build_interp_weights(parent_ny=parent_ny, parent_nx=parent_nx, child_ny=child_ny, child_nx=child_nx, **c),
        u=build_interp_weights(parent_ny=parent_ny, parent_nx=parent_nx + 1, child_ny=child_ny,
                               child_nx=child_nx + 1, **c),
        v=build_interp_weights(parent_ny=parent_ny + 1, parent_nx=parent_nx, child_ny=child_ny + 1,
                               child_nx=child_nx, **c),
        registration=registration)


# ---------------------------------------------------------------------------
# ring strips and the two-time boundary package
# ---------------------------------------------------------------------------

def field_sides_3d(field, width, side_len):
    z, ny, nx = field.shape
    xw, yw = min(width, nx), min(width, ny)
    sides = [np.moveaxis(field[:, :, :xw], 2, 0), np.moveaxis(field[:, :, nx - xw:][:, :, ::-1], 2, 0),
             np.moveaxis(field[:, :yw, :], 1, 0), np.moveaxis(field[:, ny - yw:, :][:, ::-1, :], 1, 0)]
    out = np.zeros((4, width, z, side_len))
    for s, st in enumerate(sides):
        out[s, :st.shape[0], :, :st.shape[2]] = st[:, :, :side_len]
    return out


def field_sides_2d(field, width, side_len):
    return field_sides_3d(field[None], width, side_len)


def fit(strips, z_target, side_target):
    out = strips[..., :z_target, :side_target]
    pz, ps = z_target - out.shape[-2], side_target - out.shape[-1]
    if pz > 0 or ps > 0:
        out = np.pad(out, ((0, 0), (0, 0), (0, max(pz, 0)), (0, max(ps, 0))))
    return out


def build_child_boundary_package(child, parent, weights, bdy_width=5):
    """``build_child_boundary_package`` (boundary_construction.py:360-451) on
    oracle states (SimpleNamespace leaves, ``*_bdy`` strips present)."""
    w = int(bdy_width)
    if w <= 0:
        raise ValueError("bdy_width must be positive")
    side_len = int(max(child.u_bdy.shape[-1], child.v_bdy.shape[-1]))

    def two_time(old_leaf, child_field, new_strips):
        zt, st = old_leaf.shape[-2], old_leaf.shape[-1]
        old = fit(field_sides_3d(child_field if child_field.ndim == 3 else child_field[None], w, side_len), zt, st)
        return np.stack([old, fit(new_strips, zt, st)], axis=0)

    ring = lambda f, wt: field_sides_3d(interp(f, wt) if f.ndim == 3 else interp(f, wt)[None], w, side_len)
    child_phb = child.ph_total - child.ph_perturbation
    child_pb = child.p_total - child.p_perturbation
    child_mub = child.mu_total - child.mu_perturbation
    out = SimpleNamespace(**vars(child))
    out.u_bdy = two_time(child.u_bdy, child.u, ring(parent.u, weights.u))
    out.v_bdy = two_time(child.v_bdy, child.v, ring(parent.v, weights.v))
    out.w_bdy = two_time(child.w_bdy, child.w, ring(parent.w, weights.mass))
    out.theta_bdy = two_time(child.theta_bdy, child.theta, ring(parent.theta, weights.mass))
    out.qv_bdy = two_time(child.qv_bdy, child.qv, ring(parent.qv, weights.mass))
    out.ph_bdy = two_time(child.ph_bdy, child.ph_perturbation, ring(parent.ph_perturbation, weights.mass))
    out.phb_bdy = two_time(child.phb_bdy, child_phb, field_sides_3d(child_phb, w, side_len))
    out.p_bdy = two_time(child.p_bdy, child.p_perturbation, ring(parent.p_perturbation, weights.mass))
    out.pb_bdy = two_time(child.pb_bdy, child_pb, field_sides_3d(child_pb, w, side_len))
    out.mu_bdy = two_time(child.mu_bdy, child.mu_perturbation, ring(parent.mu_perturbation, weights.mass))
    out.mub_bdy = two_time(child.mub_bdy, child_mub, field_sides_2d(child_mub, w, side_len))
    return out


# ---------------------------------------------------------------------------
# child -> parent feedback
# ---------------------------------------------------------------------------

def build_feedback_plan(*, ratio, i_parent_start, j_parent_start, parent_we, parent_sn, child_we, child_sn,
                        stagger="", spec_zone=1):
    """``build_feedback_weights`` (boundary_feedback.py:170-267): parent
    linear indices of the overlap and their child donor indices."""
    if stagger not in ("", "U", "V"):
        raise ValueError(stagger)
    r = int(ratio)
    if r <= 1:
        raise ValueError("feedback requires parent_grid_ratio > 1")
    if r % 2 == 0:
        raise NotImplementedError("even ratios")
    ipos, jpos, sz = int(i_parent_start), int(j_parent_start), int(spec_zone)
    pwe = parent_we + (1 if stagger == "U" else 0)
    psn = parent_sn + (1 if stagger == "V" else 0)
    cwe = child_we + (1 if stagger == "U" else 0)
    csn = child_sn + (1 if stagger == "V" else 0)
    istag = 0 if stagger == "U" else 1
    jstag = 0 if stagger == "V" else 1
    n_pi, n_pj = child_we // r, child_sn // r
    parent_lin, child_lin = [], []
    for cj in range(jpos + sz, jpos + n_pj - jstag - sz + 1):
        for ci in range(ipos + sz, ipos + n_pi - istag - sz + 1):
            if stagger == "":
                ni, nj = (ci - ipos) * r + r // 2 + 1, (cj - jpos) * r + r // 2 + 1
                donors = [(nj + jj - r // 2 - 1) * cwe + (ni + ii - r // 2 - 1) for jj in range(r) for ii in range(r)]
            elif stagger == "U":
                ni, nj = (ci - ipos) * r + 1, (cj - jpos) * r + r // 2 + 1
                donors = [(nj + jj - r // 2 - 1) * cwe + (ni - 1) for jj in range(r)]
            else:
                ni, nj = (ci - ipos) * r + r // 2 + 1, (cj - jpos) * r + 1
                donors = [(nj - 1) * cwe + (ni + ii - r // 2 - 1) for ii in range(r)]
            for d in donors:
                drow, dcol = divmod(d, cwe)
                if not (0 <= drow < csn and 0 <= dcol < cwe):
                    raise IndexError("feedback donor out of bounds")
            parent_lin.append((cj - 1) * pwe + (ci - 1))
            child_lin.append(donors)
    stencil = r * r if stagger == "" else r
    return SimpleNamespace(parent_lin=np.asarray(parent_lin, dtype=np.int32),
                           child_lin=np.asarray(child_lin, dtype=np.int32).reshape(-1, stencil),
                           pwe=pwe, psn=psn, cwe=cwe, csn=csn, stencil=stencil, ratio=r, stagger=stagger)


def build_smoother(*, ratio, i_parent_start, j_parent_start, child_we, child_sn, stagger=""):
    """``build_feedback_smoother`` (boundary_feedback.py:270-319)."""
    r = int(ratio)
    istag = 0 if stagger == "U" else 1
    jstag = 0 if stagger == "V" else 1
    i_lo_1, i_hi_1 = i_parent_start + 2, i_parent_start + child_we // r - 2 - istag
    j_lo_1, j_hi_1 = j_parent_start + 2, j_parent_start + child_sn // r - 2 - jstag
    i_lo, j_lo = i_lo_1 - 1, j_lo_1 - 1
    return SimpleNamespace(i_lo=max(i_lo, 0), i_hi=max(i_hi_1, i_lo), j_lo=max(j_lo, 0), j_hi=max(j_hi_1, j_lo))


def feedback_values(child, plan):
    """The overlap means (boundary_feedback.py:362-375), summed in donor order."""
    c = child if child.ndim == 3 else child[None]
    flat = c.reshape(c.shape[0], plan.csn * plan.cwe)
    g = flat[:, plan.child_lin]  # (z, npts, stencil)
    acc = g[:, :, 0].copy()
    for s in range(1, plan.stencil):
        acc = acc + g[:, :, s]
    vals = acc / float(plan.stencil)
    return vals if child.ndim == 3 else vals[0]


def apply_feedback(parent, child, plan):
    p = (parent if parent.ndim == 3 else parent[None]).copy()
    flat = p.reshape(p.shape[0], plan.psn * plan.pwe)
    v = feedback_values(child, plan)
    flat[:, plan.parent_lin] = v if v.ndim == 2 else v[None]
    out = flat.reshape(p.shape)
    return out if parent.ndim == 3 else out[0]


def sm121(field, sm):
    """``sm121_smooth`` (boundary_feedback.py:428-494): the j 1-2-1 pass into
    a copy, then the i pass over the interior from that copy."""
    i_lo, i_hi, j_lo, j_hi = sm.i_lo, sm.i_hi, sm.j_lo, sm.j_hi
    if i_hi <= i_lo or j_hi <= j_lo:
        return field
    a = field if field.ndim == 3 else field[None]
    ny, nx = a.shape[-2], a.shape[-1]
    if i_lo < 1 or i_hi > nx - 1 or j_lo < 1 or j_hi > ny - 1:
        i_lo, i_hi, j_lo, j_hi = max(i_lo, 1), min(i_hi, nx - 1), max(j_lo, 1), min(j_hi, ny - 1)
        if i_hi <= i_lo or j_hi <= j_lo:
            return field
    cnew = a.copy()
    cnew[:, j_lo:j_hi, i_lo:i_hi] = 0.25 * (a[:, j_lo + 1:j_hi + 1, i_lo:i_hi] + 2.0 * a[:, j_lo:j_hi, i_lo:i_hi]
                                            + a[:, j_lo - 1:j_hi - 1, i_lo:i_hi])
    out = a.copy()
    out[:, j_lo:j_hi, i_lo:i_hi] = 0.25 * (cnew[:, j_lo:j_hi, i_lo + 1:i_hi + 1] + 2.0 * cnew[:, j_lo:j_hi, i_lo:i_hi]
                                           + cnew[:, j_lo:j_hi, i_lo - 1:i_hi - 1])
    return out if field.ndim == 3 else out[0]


def build_state_feedback_plans(*, ratio, i_parent_start, j_parent_start, parent_nx, parent_ny, child_nx, child_ny,
                               spec_zone=1, smooth_option=1):
    c = dict(ratio=ratio, i_parent_start=i_parent_start, j_parent_start=j_parent_start, parent_we=parent_nx,
             parent_sn=parent_ny, child_we=child_nx, child_sn=child_ny, spec_zone=spec_zone)
    sc = dict(ratio=ratio, i_parent_start=i_parent_start, j_parent_start=j_parent_start, child_we=child_nx,
              child_sn=child_ny)
    return SimpleNamespace(mass=build_feedback_plan(stagger="", **c), u=build_feedback_plan(stagger="U", **c),
                           v=build_feedback_plan(stagger="V", **c), mass_smooth=build_smoother(stagger="", **sc),
                           u_smooth=build_smoother(stagger="U", **sc), v_smooth=build_smoother(stagger="V", **sc),
                           smooth_option=int(smooth_option))


MOIST_FB = ("qc", "qr", "qi", "qs", "qg")


def apply_state_feedback(parent, child, plans, feedback=True):
    """``apply_state_feedback`` (boundary_feedback.py:509-592) for the State
    leaves this build carries (u, v, w, theta, qv, p', ph', mu', qc..qg)."""
    if not feedback:
        return parent
    smooth = plans.smooth_option != 0

    def fb(p, c, plan, sm):
        out = apply_feedback(p, c, plan)
        return sm121(out, sm) if smooth else out

    out = SimpleNamespace(**vars(parent))
    out.u = fb(parent.u, child.u, plans.u, plans.u_smooth)
    out.v = fb(parent.v, child.v, plans.v, plans.v_smooth)
    out.w = fb(parent.w, child.w, plans.mass, plans.mass_smooth)
    out.theta = fb(parent.theta, child.theta, plans.mass, plans.mass_smooth)
    out.qv = fb(parent.qv, child.qv, plans.mass, plans.mass_smooth)
    out.p_perturbation = fb(parent.p_perturbation, child.p_perturbation, plans.mass, plans.mass_smooth)
    out.ph_perturbation = fb(parent.ph_perturbation, child.ph_perturbation, plans.mass, plans.mass_smooth)
    out.mu_perturbation = fb(parent.mu_perturbation, child.mu_perturbation, plans.mass, plans.mass_smooth)
    out.p_total = (parent.p_total - parent.p_perturbation) + out.p_perturbation
    out.ph_total = (parent.ph_total - parent.ph_perturbation) + out.ph_perturbation
    out.mu_total = (parent.mu_total - parent.mu_perturbation) + out.mu_perturbation
    for q in MOIST_FB:
        pv, cv = getattr(parent, q, None), getattr(child, q, None)
        if pv is not None and cv is not None:
            setattr(out, q, fb(pv, cv, plans.mass, plans.mass_smooth))
    return out
