"""The RK3 step as a PyTorch operator: ``torch.ops.wrfgpu.rk3_step``.

A ``torch.library`` custom op over the C ABI (``wrfgpu_rk3_step`` /
``wrfgpu_rk3_step_device_lead``), so the step composes with other torch ops,
runs on the current CUDA stream and has a fake (meta) implementation for
shape propagation.  It is the torch-side form of the reference's
``_rk_scan_step`` (runtime/operational_mode.py:3319-3534); the statics of the
step (the namelist fields and the metric arrays) are bound once by
``register_plan`` and passed to the op as an integer handle, because a
namelist is not a tensor.

Arguments of ``torch.ops.wrfgpu.rk3_step(fields, strips, mudf, lead_seconds,
plan)``:

* ``fields``: the 16 state leaves in ``STEP_FIELDS`` order (u, v, w, theta,
  p_total, p_perturbation, ph_total, ph_perturbation, mu_total,
  mu_perturbation, qv, qc, qr, qi, qs, qg), contiguous float64 on the device;
* ``strips``: the boundary strips in ``STRIP_FIELDS`` order (u_bdy, v_bdy,
  theta_bdy, ph_bdy, mu_bdy, w_bdy), or an empty list without boundaries;
* ``mudf``: the carry's mudf (ny, nx);
* ``lead_seconds``: a one-element float64 device tensor (the traced clock),
  or None (no lead: boundary forcing off);
* ``plan``: the handle from ``register_plan``.

Returns the 16 new state leaves followed by the 13 carry outputs in
``CARRY_OUT`` order.
"""

from __future__ import annotations

import itertools

import torch

from . import dycore

STEP_FIELDS = ("u", "v", "w", "theta", "p_total", "p_perturbation", "ph_total", "ph_perturbation", "mu_total",
               "mu_perturbation", "qv", "qc", "qr", "qi", "qs", "qg")
STRIP_FIELDS = ("u_bdy", "v_bdy", "theta_bdy", "ph_bdy", "mu_bdy", "w_bdy")
CARRY_OUT = ("t_2ave", "ww", "mudf", "muave", "muts", "ph_tend", "u_save", "v_save", "w_save", "t_save", "ph_save",
             "mu_save", "ww_save")

_PLANS: dict[int, dycore.Stepper] = {}
_NEXT = itertools.count(1)


def register_plan(namelist: dycore.OperationalNamelist, device="cuda") -> int:
    """Validate ``namelist`` for the op and bind its statics; returns the
    handle.  Raises ``NotImplementedError`` for unsupported configurations,
    as the reference raises at trace time."""
    stp = dycore.Stepper(namelist, device=device, own_workspace=False)
    h = next(_NEXT)
    _PLANS[h] = stp
    return h


def release_plan(plan: int) -> None:
    _PLANS.pop(int(plan), None)


def _carry_shapes(fields):
    u, w, theta, mu = fields[0], fields[2], fields[3], fields[8]
    return dict(t_2ave=theta, ww=w, mudf=mu, muave=mu, muts=mu, ph_tend=w, u_save=u, v_save=fields[1], w_save=w,
                t_save=theta, ph_save=w, mu_save=mu, ww_save=w)


@torch.library.custom_op("wrfgpu::rk3_step", mutates_args=())
def rk3_step(fields: list[torch.Tensor], strips: list[torch.Tensor], mudf: torch.Tensor,
             lead_seconds: torch.Tensor | None, plan: int) -> list[torch.Tensor]:
    stp = _PLANS.get(int(plan))
    if stp is None:
        raise ValueError(f"wrfgpu::rk3_step: unknown plan {plan} (use register_plan)")
    if len(fields) != len(STEP_FIELDS):
        raise ValueError(f"wrfgpu::rk3_step: {len(STEP_FIELDS)} state fields expected, got {len(fields)}")
    if strips and len(strips) != len(STRIP_FIELDS):
        raise ValueError(f"wrfgpu::rk3_step: {len(STRIP_FIELDS)} strips or none expected, got {len(strips)}")
    kw = dict(zip(STEP_FIELDS, fields))
    if strips:
        kw.update(zip(STRIP_FIELDS, strips))
    carry = dycore.OperationalCarry(state=dycore.State(**kw), mudf=mudf)
    out = stp.alloc_carry(carry)
    stp.step_into(carry, out, lead_seconds=lead_seconds)
    return [getattr(out.state, n) for n in STEP_FIELDS] + [getattr(out, n) for n in CARRY_OUT]


@rk3_step.register_fake
def _rk3_step_fake(fields, strips, mudf, lead_seconds, plan):
    like = _carry_shapes(fields)
    return [torch.empty_like(f) for f in fields] + [torch.empty_like(like[n]) for n in CARRY_OUT]


def rk_scan_step(carry: dycore.OperationalCarry, plan: int, lead_seconds=None) -> dycore.OperationalCarry:
    """``dycore.rk_scan_step`` through the torch operator: ``carry`` must hold
    all six moisture species; ``lead_seconds`` None, a float or a one-element
    float64 device tensor."""
    s = carry.state
    fields = [getattr(s, n) for n in STEP_FIELDS]
    if any(f is None for f in fields):
        raise ValueError("the torch operator needs every state leaf, the six moisture species included")
    strips = [getattr(s, n) for n in STRIP_FIELDS]
    if all(t is None for t in strips):
        strips = []
    elif any(t is None for t in strips):
        raise ValueError("the torch operator takes all six boundary strips (u, v, theta, ph, mu, w) or none")
    if isinstance(lead_seconds, (int, float)):
        lead_seconds = torch.full((1,), float(lead_seconds), dtype=torch.float64, device=s.u.device)
    mudf = carry.mudf if carry.mudf is not None else torch.zeros_like(s.mu_total)
    res = torch.ops.wrfgpu.rk3_step(fields, strips, mudf, lead_seconds, int(plan))
    st = dycore.State(**dict(zip(STEP_FIELDS, res[:len(STEP_FIELDS)])),
                      **{n: getattr(s, n) for n in dycore._LEAVES})
    return dycore.OperationalCarry(state=st, **dict(zip(CARRY_OUT, res[len(STEP_FIELDS):])),
                                   base_state=carry.base_state)
