"""The drop-in boundary with the reference's traced clock, and the torch op.

* ``wrfgpu_rk3_step_device_lead``: one CUDA graph of the step captured once
  and replayed for three steps while only the device-resident lead changes
  (the reference computes ``lead_seconds = step_index * dt`` inside its jitted
  loop, runtime/operational_mode.py:4929), on a specified case with drifting
  strips under the boundary cadence; every replay matches the oracle's step
  at that lead to 1e-12.
* ``torch.ops.wrfgpu.rk3_step`` (a ``torch.library`` custom op) gives the
  same bits as ``dycore.rk_scan_step``.
* ``forecast_step`` with a device step index equals the host-clock form.
* ``rk_scan_step``'s prepared-step cache is bounded and keyed by content.
"""

from __future__ import annotations

from dataclasses import replace
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import dycore as D
from tests import parity_util as P
from tests.test_gpu_parity import _tol
from wrf_gpu_b200 import cases, dycore, torch_ops

pytestmark = pytest.mark.gpu


def _drifting_case():
    case = cases.real_like_moist(40, 24, 12, hmax=800.0, specified=True, bdy_noise=True)
    # strips 20 s apart, so the 6 s steps interpolate at a different weight each step
    case.controls.update(specified_bdy_cadence=True, update_cadence_s=20.0)
    return case


def _copy_in(dst: dycore.OperationalCarry, state, mudf):
    for f in P.STATE_KEYS:
        getattr(dst.state, f).copy_(torch.as_tensor(getattr(state, f), device="cuda"))
    dst.mudf.copy_(torch.as_tensor(mudf, device="cuda"))


def test_graph_replay_with_device_lead_matches_oracle(cuda_ready):
    case = _drifting_case()
    nl = dycore.OperationalNamelist.from_case(case)
    stp = dycore.Stepper(nl)
    a = dycore.carry_from_case(case)
    b = stp.alloc_carry(a)
    lead = torch.zeros(1, dtype=torch.float64, device="cuda")
    stp.step_into(a, b, lead_seconds=lead)  # warm-up outside the capture
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        stp.step_into(a, b, lead_seconds=lead)
    onl = P.oracle_namelist(case)
    carry = SimpleNamespace(state=D.copy_state(case.state), mudf=case.mudf.copy())
    for n in range(3):
        t = n * onl.dt_s
        ora = D.rk_scan_step(carry, onl, lead_seconds=t)
        _copy_in(a, carry.state, carry.mudf)
        lead.fill_(t)
        graph.replay()
        torch.cuda.synchronize()
        errs = P.compare(b, ora)
        bad = {k: v for k, v in errs.items() if not v <= _tol(k)}
        assert not bad, f"replay {n} (lead {t} s): {bad}"
        carry = SimpleNamespace(state=ora.state, mudf=ora.mudf)
    del graph


def test_device_lead_equals_host_lead(cuda_ready):
    case = _drifting_case()
    nl = dycore.OperationalNamelist.from_case(case)
    carry = dycore.carry_from_case(case)
    for t in (0.0, 6.0, 27.0):
        host = dycore.rk_scan_step(carry, nl, lead_seconds=t)
        dev = dycore.rk_scan_step(carry, nl, lead_seconds=torch.tensor([t], dtype=torch.float64, device="cuda"))
        torch.cuda.synchronize()
        for f in P.STATE_KEYS:
            assert torch.equal(getattr(host.state, f), getattr(dev.state, f)), (t, f)


def test_torch_op_matches_shim(cuda_ready):
    case = cases.real_like_moist(24, 20, 14, hmax=800.0, specified=True)
    nl = dycore.OperationalNamelist.from_case(case)
    carry = dycore.carry_from_case(case)
    plan = torch_ops.register_plan(nl)
    try:
        via_op = torch_ops.rk_scan_step(carry, plan, lead_seconds=0.0)
        via_shim = dycore.rk_scan_step(carry, nl, lead_seconds=0.0)
        torch.cuda.synchronize()
        for f in P.STATE_KEYS:
            assert torch.equal(getattr(via_op.state, f), getattr(via_shim.state, f)), f
        for f in P.CARRY_KEYS:
            assert torch.equal(getattr(via_op, f), getattr(via_shim, f)), f
    finally:
        torch_ops.release_plan(plan)


def test_forecast_step_device_clock_equals_host_clock(cuda_ready):
    case = cases.with_full_leaves(cases.real_like_moist(32, 24, 12, hmax=800.0, specified=True, bdy_noise=True),
                                  rng=np.random.default_rng(3))
    case.controls.update(specified_bdy_cadence=True, update_cadence_s=20.0)
    nl = dycore.OperationalNamelist.from_case(case)
    carry = dycore.carry_from_case(case)
    for idx in (0, 2, 5):
        h, hd = dycore.forecast_step(carry, nl, idx)
        d, dd = dycore.forecast_step(carry, nl, torch.tensor([idx], dtype=torch.int64, device="cuda"))
        torch.cuda.synchronize()
        for f in P.STATE_KEYS:
            assert torch.equal(getattr(h.state, f), getattr(d.state, f)), (idx, f)
        assert int(hd["theta_limited_cell_count"]) == int(dd["theta_limited_cell_count"])


def test_prepared_step_cache_is_bounded_and_keyed_by_content(cuda_ready):
    case = cases.real_like_moist(12, 10, 6, hmax=300.0, specified=False)
    nl = dycore.OperationalNamelist.from_case(case)
    carry = dycore.carry_from_case(case)
    dycore._PLANS.clear()
    dycore.rk_scan_step(carry, nl, lead_seconds=0.0)
    dycore.rk_scan_step(carry, replace(nl), lead_seconds=0.0)  # a new namelist object, same content
    assert len(dycore._PLANS) == 1
    for k in range(2 * dycore._PLAN_CAPACITY):
        dycore.rk_scan_step(carry, replace(nl, epssm=0.1 + 0.01 * k), lead_seconds=0.0)
    torch.cuda.synchronize()
    assert len(dycore._PLANS) == dycore._PLAN_CAPACITY
