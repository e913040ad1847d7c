"""Batched domains and the tile-shape tuner.

* ``wrfgpu_rk3_step_batched`` advances members of different sizes and
  configurations (a moist specified-boundary domain, a periodic one, a dry
  warm bubble) in one call; each member's result must equal, bit for bit, the
  same member stepped alone with ``wrfgpu_rk3_step``, both directly and when
  the batched call is captured in a CUDA graph and replayed.
* ``wrfgpu_autotune`` returns valid tile shapes, and a step with any tile
  shape is bit-identical to the default (the shapes only change how the work
  is laid out on the GPU, not the arithmetic).
"""

from __future__ import annotations

import pytest
import torch

from wrf_gpu_b200 import cases, dycore

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "theta", "p_perturbation", "ph_perturbation", "mu_perturbation", "qv")


def _members():
    return [cases.real_like_moist(40, 36, 20, hmax=800.0, specified=True),
            cases.real_like_moist(24, 20, 14, hmax=600.0, specified=False, seed=3),
            cases.warm_bubble_3d(32, 24, 16)]


def _same(a, b):
    for f in FIELDS:
        x, y = getattr(a.state, f), getattr(b.state, f)
        if x is None and y is None:
            continue
        assert torch.equal(x, y), f
    assert torch.equal(a.ww, b.ww) and torch.equal(a.mudf, b.mudf)


def test_batched_equals_individual_steps(cuda_ready):
    members = _members()
    nls = [dycore.OperationalNamelist.from_case(c) for c in members]
    carries = [dycore.carry_from_case(c) for c in members]
    bs = dycore.BatchStepper(nls)
    outs_b = bs.alloc_carries(carries)
    bs.step_into(carries, outs_b, lead_seconds=0.0)
    singles = []
    for nl, c in zip(nls, carries):
        st = dycore.Stepper(nl)
        o = st.alloc_carry(c)
        st.step_into(c, o, lead_seconds=0.0)
        singles.append(o)
    torch.cuda.synchronize()
    for a, b in zip(outs_b, singles):
        _same(a, b)

    # the batched call captured in one CUDA graph (parallel branches) and replayed
    outs_g = bs.alloc_carries(carries)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        bs.step_into(carries, outs_g, lead_seconds=0.0)  # first call on this stream outside capture
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        bs.step_into(carries, outs_g, lead_seconds=0.0)
    for o in outs_g:
        o.state.u.zero_()
    graph.replay()
    torch.cuda.synchronize()
    for a, b in zip(outs_g, singles):
        _same(a, b)
    del graph


def test_autotune_picks_valid_shapes_and_results_do_not_depend_on_them(cuda_ready):
    case = cases.real_like_moist(64, 48, 20, hmax=800.0, specified=True)
    nl = dycore.OperationalNamelist.from_case(case)
    carry = dycore.carry_from_case(case)
    st = dycore.Stepper(nl)
    ref = st.alloc_carry(carry)
    st.step_into(carry, ref, lead_seconds=0.0)
    scratch = st.alloc_carry(carry)
    kc, lanes, width = st.autotune(carry, scratch)
    assert kc in (0, 5, 10, 25)
    assert lanes in (0, 8, 13, 16)
    assert width in (0, 16, 32)
    for kc_, lanes_, width_ in ((kc, lanes, width), (5, 8, 16), (25, 16, 32), (10, 13, 16), (10, 16, 16)):
        st.params.march_levels, st.params.column_lanes, st.params.column_width = kc_, lanes_, width_
        o = st.alloc_carry(carry)
        st.step_into(carry, o, lead_seconds=0.0)
        torch.cuda.synchronize()
        _same(o, ref)


def test_batched_members_match_the_oracle(cuda_ready):
    """Each member of one batched call (uneven sizes, moist specified, moist
    periodic, dry warm bubble) against the oracle's step of the same input,
    at the per-step parity tolerance."""
    from types import SimpleNamespace

    from oracle import dycore as D
    from tests import parity_util as P

    members = _members()
    nls = [dycore.OperationalNamelist.from_case(c) for c in members]
    carries = [dycore.carry_from_case(c) for c in members]
    bs = dycore.BatchStepper(nls)
    outs = bs.alloc_carries(carries)
    bs.step_into(carries, outs, lead_seconds=0.0)
    torch.cuda.synchronize()
    # the warm bubble starts at rest: after one step its winds and the mass
    # diagnostics are at the float64 noise floor, where one-ulp pow()
    # differences are ~1e-12..1e-11 relative (the warm-bubble parity bound)
    rest = ("u", "v", "w", "u_save", "v_save", "w_save", "mudf", "muave", "ww", "ww_save", "ph_tend",
            "p_perturbation")
    for n, (case, out) in enumerate(zip(members, outs)):
        ora = D.rk_scan_step(SimpleNamespace(state=D.copy_state(case.state), mudf=case.mudf.copy()),
                             P.oracle_namelist(case), lead_seconds=0.0)
        for k, e in P.compare(out, ora).items():
            if n == 2 and k in rest:
                tol = 1.0e-10
            else:
                tol = 5.0e-12 if k in ("mudf", "muave", "p_perturbation") else 1.0e-12
            assert e <= tol, (n, k, e)
