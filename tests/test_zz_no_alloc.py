"""The step entry point that allocates nothing, against the ordinary one.

``wrfgpu_rk3_step_static_workspace`` serves callers that cannot allocate
device memory: a host framework whose own pool owns the GPU's memory, or a
host model that calls one routine per step with a fixed argument list and has
nowhere to keep a workspace.  Its scratch is a fixed 32 MiB array held by the
library on each GPU, shared by every call and keeping the previous call's
contents.  This test runs two steps in a row through it and the same two steps
through ``wrfgpu_rk3_step`` (whose workspace is filled with NaN bytes first, so
a scratch value read before it is written would show), and requires the
outputs to agree within the parity tolerance of the other GPU tests.  It also
checks that a grid too large for the array is refused with a clear error.

The file name makes pytest collect it last; it passes alone in a fresh
process and after the other tests.
"""

from __future__ import annotations

import ctypes

import pytest
import torch

from wrf_gpu_b200 import _capi, cases, dycore

pytestmark = pytest.mark.gpu

TOL = 1.0e-12


def _structs(carry, out, nl):
    """C structs for one step from ``carry`` into ``out`` (as Stepper.step_into builds them)."""
    p = dycore._ptr
    s, o = carry.state, out.state
    ins = _capi.StepInputs()
    for n in dycore.STATE_FIELDS:
        setattr(ins, n, p(getattr(s, n)))
    for k, n in enumerate(dycore.MOIST):
        ins.q[k] = p(getattr(s, n))
    ins.mudf = p(carry.mudf)
    t = nl.tendencies
    ins.base_u, ins.base_v, ins.base_w = p(t.u), p(t.v), p(t.w)
    ins.base_theta, ins.base_mu = p(t.theta), p(t.mu)
    if nl.run_boundary and s.u_bdy is not None:
        ins.u_bdy, ins.v_bdy = p(s.u_bdy), p(s.v_bdy)
        ins.bdy_ntime, _, ins.bdy_width, _, ins.bdy_side_len = s.u_bdy.shape
    outs = _capi.StepOutputs()
    for n in dycore.STATE_FIELDS:
        setattr(outs, n, p(getattr(o, n)))
    for k, n in enumerate(dycore.MOIST):
        outs.q[k] = p(getattr(o, n))
    for n in dycore.CARRY_FIELDS:
        setattr(outs, n, p(getattr(out, n)))
    return ins, outs


def _fields(carry):
    d = {n: getattr(carry.state, n) for n in dycore.STATE_FIELDS + tuple(dycore.MOIST)}
    d.update({n: getattr(carry, n) for n in dycore.CARRY_FIELDS})
    return d


def _rel(a, b):
    den = float(b.abs().max())
    return float((a - b).abs().max()) / (den if den > 0.0 else 1.0)


def test_static_workspace_matches_caller_workspace_two_steps(cuda_ready):
    case = cases.real_like_moist(24, 20, 14, hmax=800.0, specified=True)
    nl = dycore.OperationalNamelist.from_case(case)
    stp = dycore.Stepper(nl)
    lib = stp.lib
    need = ctypes.c_size_t(0)
    _capi.check(lib.wrfgpu_step_workspace_size(ctypes.byref(stp.params), ctypes.byref(need)))
    assert need.value <= _capi.WRFGPU_STATIC_WORKSPACE_BYTES
    stream = torch.cuda.current_stream()

    start = dycore.carry_from_case(case)
    ref_prev, new_prev = start, start
    for n in range(2):
        lead = n * nl.dt_s
        ref = stp.alloc_carry(start)
        stp.workspace.fill_(0xFF)  # NaN bytes: a read-before-write would surface
        stp.step_into(ref_prev, ref, lead_seconds=lead)

        new = stp.alloc_carry(start)
        ins, outs = _structs(new_prev, new, nl)
        rc = lib.wrfgpu_rk3_step_static_workspace(ctypes.byref(stp.params), ctypes.byref(stp.metrics),
                                                  ctypes.byref(ins), ctypes.byref(outs), float(lead),
                                                  ctypes.c_void_p(stream.cuda_stream))
        _capi.check(rc)
        torch.cuda.synchronize()
        a, b = _fields(new), _fields(ref)
        for k in b:
            assert torch.isfinite(b[k]).all(), f"step {n}: caller-workspace {k} not finite"
            err = _rel(a[k], b[k])
            assert err <= TOL, f"step {n}: {k} differs by {err:.3e}"
        ref_prev, new_prev = ref, new


def test_static_workspace_rejects_a_grid_that_does_not_fit(cuda_ready):
    case = cases.real_like_moist(24, 20, 14, hmax=800.0, specified=True)
    nl = dycore.OperationalNamelist.from_case(case)
    stp = dycore.Stepper(nl)
    lib = stp.lib
    big = dycore.step_params(nl)
    big.nx, big.ny, big.nz = 433, 433, 50
    need = ctypes.c_size_t(0)
    _capi.check(lib.wrfgpu_step_workspace_size(ctypes.byref(big), ctypes.byref(need)))
    assert need.value > _capi.WRFGPU_STATIC_WORKSPACE_BYTES
    ins, outs = _capi.StepInputs(), _capi.StepOutputs()
    rc = lib.wrfgpu_rk3_step_static_workspace(ctypes.byref(big), ctypes.byref(stp.metrics), ctypes.byref(ins),
                                              ctypes.byref(outs), float("nan"),
                                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _capi.WRFGPU_ERR_WORKSPACE
    msg = lib.wrfgpu_last_error_string().decode()
    assert "workspace" in msg and str(need.value) in msg
