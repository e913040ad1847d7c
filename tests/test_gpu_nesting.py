"""Nest coupling on the GPU against the oracle: the child boundary package
(every leaf, both times), whole-field interpolation of each staggering and
the two-way state feedback with its sm121 smoother, for the sint and
node-aligned registrations and a nest whose overlap reaches the parent's
edge (the smoother's interior clamp).  The GPU evaluates the same gathers,
means (summed in donor order) and blends, so the results are bit for bit
the oracle's."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import nesting as N
from tests.test_oracle_nesting import CNX, CNY, IPOS, JPOS, PNX, PNY, RATIO, nest_pair
from wrf_gpu_b200 import dycore, nesting

pytestmark = pytest.mark.gpu


def _dev_state(s):
    return dycore.State.from_host(s)


@pytest.mark.parametrize("registration", ["sint", "bilinear"])
def test_boundary_package_matches_oracle(cuda_ready, registration):
    child, parent = nest_pair(5)
    g = lambda nx, ny: SimpleNamespace(nx=nx, ny=ny)
    w_dev = nesting.build_nest_force_weights(parent_grid_ratio=RATIO, i_parent_start=IPOS, j_parent_start=JPOS,
                                             parent_grid=g(PNX, PNY), child_grid=g(CNX, CNY),
                                             registration=registration)
    w_ora = N.build_nest_force_weights(ratio=RATIO, i_parent_start=IPOS, j_parent_start=JPOS, parent_ny=PNY,
                                       parent_nx=PNX, child_ny=CNY, child_nx=CNX, registration=registration)
    got = nesting.build_child_boundary_package(_dev_state(child), _dev_state(parent), w_dev)
    want = N.build_child_boundary_package(child, parent, w_ora)
    torch.cuda.synchronize()
    for leaf in nesting.FORCED_LEAVES:
        np.testing.assert_array_equal(getattr(got, leaf).cpu().numpy(), getattr(want, leaf), err_msg=leaf)
    for stag, f in (("mass", parent.theta), ("u", parent.u), ("v", parent.v), ("mass", parent.mu_perturbation)):
        wo = {"mass": w_ora.mass, "u": w_ora.u, "v": w_ora.v}[stag]
        out = nesting.interp_parent_field_to_child(torch.as_tensor(f, device="cuda"), w_dev, staggering=stag)
        np.testing.assert_array_equal(out.cpu().numpy(), N.interp(f, wo), err_msg=stag)


@pytest.mark.parametrize("ipos,jpos,smooth", [(IPOS, JPOS, 1), (IPOS, JPOS, 0), (1, 1, 1)])
def test_state_feedback_matches_oracle(cuda_ready, ipos, jpos, smooth):
    child, parent = nest_pair(6)
    g = lambda nx, ny: SimpleNamespace(nx=nx, ny=ny)
    w_dev = nesting.build_state_feedback_weights(parent_grid_ratio=RATIO, i_parent_start=ipos, j_parent_start=jpos,
                                                 parent_grid=g(PNX, PNY), child_grid=g(CNX, CNY),
                                                 smooth_option=smooth)
    plans = N.build_state_feedback_plans(ratio=RATIO, i_parent_start=ipos, j_parent_start=jpos, parent_nx=PNX,
                                         parent_ny=PNY, child_nx=CNX, child_ny=CNY, smooth_option=smooth)
    got = nesting.apply_state_feedback(_dev_state(parent), _dev_state(child), w_dev)
    want = N.apply_state_feedback(parent, child, plans)
    torch.cuda.synchronize()
    for f in ("u", "v", "w", "theta", "qv", "qc", "qr", "p_perturbation", "ph_perturbation", "mu_perturbation",
              "p_total", "ph_total", "mu_total"):
        np.testing.assert_array_equal(getattr(got, f).cpu().numpy(), getattr(want, f), err_msg=f)
