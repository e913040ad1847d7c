"""A two-level nest advanced by WRF's integrate recursion on the GPU
(``nesting.NestTower``) against the same recursion over the oracle: the 3:1
child takes three own steps per parent step with its boundary package rebuilt
from the just-advanced parent, with and without two-way feedback.  The
parent runs under the specified boundary cadence, the child as a nested
domain (force_geopotential off) whose strips are interpolated over its
parent's step."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import dycore as D
from oracle import nesting as N
from tests import parity_util as P
from wrf_gpu_b200 import cases, dycore, nesting

pytestmark = pytest.mark.gpu

RATIO, IPOS, JPOS = 3, 3, 2
PNX, PNY, CNX, CNY, NZ = 24, 20, 27, 24, 10
PDT = 9.0


def tower_cases():
    parent = cases.with_full_leaves(cases.real_like_moist(PNX, PNY, NZ, dx=3000.0, dt=PDT, hmax=100.0,
                                                          specified=True))
    parent.controls["specified_bdy_cadence"] = True
    child = cases.with_full_leaves(cases.real_like_moist(CNX, CNY, NZ, dx=1000.0, dt=PDT / RATIO, hmax=100.0,
                                                         specified=True, seed=1))
    child.controls.update(force_geopotential=False, update_cadence_s=PDT, nested_ph_relax=True)
    return parent, child


def oracle_tower(parent, child, parent_steps, feedback):
    nls = {"p": P.oracle_namelist(parent), "c": P.oracle_namelist(child)}
    st = {"p": SimpleNamespace(state=D.copy_state(parent.state), mudf=parent.mudf.copy()),
          "c": SimpleNamespace(state=D.copy_state(child.state), mudf=child.mudf.copy())}
    fw = N.build_nest_force_weights(ratio=RATIO, i_parent_start=IPOS, j_parent_start=JPOS, parent_ny=PNY,
                                    parent_nx=PNX, child_ny=CNY, child_nx=CNX)
    fb = N.build_state_feedback_plans(ratio=RATIO, i_parent_start=IPOS, j_parent_start=JPOS, parent_nx=PNX,
                                      parent_ny=PNY, child_nx=CNX, child_ny=CNY)

    def advance(name, local):
        nl = nls[name]
        lead = local * nl.dt_s
        origin = st[name].state
        nxt = D.rk_scan_step(st[name], nl, lead_seconds=lead)
        spec_only = nl.specified_bdy_cadence and nl.run_boundary and not nl.bc_ideal and nl.force_geopotential
        s, _ = D.step_epilogue(nxt.state, origin, lead, nl.dt_s, nl, run_boundary=True, dry_spec_only=spec_only)
        st[name] = SimpleNamespace(state=s, mudf=nxt.mudf)

    for lp in range(1, parent_steps + 1):
        advance("p", lp)
        pkg = N.build_child_boundary_package(st["c"].state, st["p"].state, fw)
        st["c"] = SimpleNamespace(state=pkg, mudf=st["c"].mudf)
        for lc in range(1, RATIO + 1):
            advance("c", lc)
        if feedback:
            st["p"] = SimpleNamespace(state=N.apply_state_feedback(st["p"].state, st["c"].state, fb),
                                      mudf=st["p"].mudf)
    return st


# The child starts from its own state and adjusts to the parent's boundary
# package, which amplifies rounding differences: the oracle tower itself moves
# by up to ~1e-6 relative (child w) when both domains' initial theta moves by
# one ulp.  The bound is therefore per field 10x that one-ulp spread (1e-10
# where the spread is smaller).
TOWER_FACTOR, TOWER_FLOOR = 10.0, 1.0e-10


@pytest.mark.parametrize("feedback", [False, True])
def test_nest_tower_matches_oracle(cuda_ready, feedback):
    parent, child = tower_cases()
    want = oracle_tower(parent, child, 2, feedback)
    parent_u, child_u = tower_cases()
    parent_u.state.theta = np.nextafter(parent_u.state.theta, np.inf)
    child_u.state.theta = np.nextafter(child_u.state.theta, np.inf)
    spread_run = oracle_tower(parent_u, child_u, 2, feedback)
    nls = {"p": dycore.OperationalNamelist.from_case(parent), "c": dycore.OperationalNamelist.from_case(child)}
    grids = {"p": SimpleNamespace(nx=PNX, ny=PNY), "c": SimpleNamespace(nx=CNX, ny=CNY)}
    tower = nesting.NestTower(["p", "c"], [nesting.NestEdge("p", "c", RATIO, IPOS, JPOS)], nls, grids,
                              feedback=feedback)
    got = tower.run({"p": dycore.carry_from_case(parent), "c": dycore.carry_from_case(child)}, 2)
    torch.cuda.synchronize()
    fields = ("u", "v", "w", "theta", "p_perturbation", "ph_perturbation", "mu_perturbation", "qv")
    for name in ("p", "c"):
        errs = {f: P.rel_err(getattr(got[name].state, f).cpu().numpy(), getattr(want[name].state, f)) for f in fields}
        spread = {f: P.rel_err(getattr(spread_run[name].state, f), getattr(want[name].state, f)) for f in fields}
        print(name, "feedback" if feedback else "one-way", {k: f"{v:.1e}" for k, v in errs.items()},
              "one-ulp spread", {k: f"{v:.1e}" for k, v in spread.items()})
        assert all(np.isfinite(getattr(want[name].state, f)).all() for f in errs)
        bad = {k: (v, spread[k]) for k, v in errs.items() if not v <= max(TOWER_FACTOR * spread[k], TOWER_FLOOR)}
        assert not bad, (name, bad)
