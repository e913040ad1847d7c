"""The forecast step's epilogue on the GPU (``wrfgpu_step_epilogue`` /
``dycore.step_epilogue``: runtime/operational_mode.py:4950-4983 without
physics) against the oracle's ``step_epilogue``: a step output with planted
offenders (non-finite and out-of-envelope theta, an out-of-range and a
negative mixing ratio, a non-finite column mass, an infinite wind) and an
origin state, through the guards + boundary pass, the boundary pass alone,
the guards alone and the specified cadence's ring-0 pass."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import dycore as D
from tests import parity_util as P
from wrf_gpu_b200 import cases, dycore

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "theta", "qv", "qc", "qr", "qi", "qs", "qg", "p_total", "p_perturbation", "ph_total",
          "ph_perturbation", "mu_total", "mu_perturbation")


def _pair(plant=True):
    case = cases.real_like_moist(26, 18, 8, hmax=600.0, specified=True, bdy_noise=True)
    origin = D.copy_state(case.state)
    rng = np.random.default_rng(5)
    P.attach_lbc_leaves(origin, rng)
    cand = D.copy_state(origin)
    cand.theta = cand.theta + rng.standard_normal(cand.theta.shape)
    cand.mu_perturbation = cand.mu_perturbation + 10.0 * rng.standard_normal(cand.mu_perturbation.shape)
    cand.mu_total = cand.mu_total + (cand.mu_perturbation - origin.mu_perturbation)
    if plant:
        cand.theta[2, 1, 1], cand.theta[3, 8, 9], cand.theta[5, 9, 20] = np.nan, 1200.0, -4.0
        cand.qv[1, 8, 8], cand.qc[0, 0, 0], cand.qr[4, 2, 3] = 0.2, -1.0, np.inf
        cand.mu_perturbation[7, 7], cand.mu_total[7, 7] = np.nan, np.nan
        cand.mu_total[9, 12] = 0.5
        cand.u[0, 8, 8], cand.w[3, 1, 2] = np.inf, np.nan
    return case, origin, cand


@pytest.mark.parametrize("run_boundary,disable_guards,cadence", [
    (True, False, False), (True, True, False), (False, False, False), (True, False, True)])
def test_epilogue_matches_oracle(cuda_ready, run_boundary, disable_guards, cadence):
    case, origin, cand = _pair()
    nlo = SimpleNamespace(update_cadence_s=3600.0, spec_zone=1, relax_zone=4, force_geopotential=True)
    want, wd = D.step_epilogue(cand, origin, 1800.0, case.controls["dt_s"], nlo, run_boundary=run_boundary,
                               disable_guards=disable_guards, dry_spec_only=cadence)
    nl = dycore.OperationalNamelist.from_case(case, run_boundary=run_boundary, disable_guards=disable_guards,
                                              specified_bdy_cadence=cadence, bc_source="wrfbdy")
    got, gd = dycore.step_epilogue(dycore.State.from_host(cand), dycore.State.from_host(origin), 1800.0, nl)
    torch.cuda.synchronize()
    for f in FIELDS:
        g, w = getattr(got, f).cpu().numpy(), getattr(want, f)
        np.testing.assert_array_equal(np.isfinite(g), np.isfinite(w), err_msg=f)
        fin = np.isfinite(w)
        err = P.rel_err(g[fin], w[fin])
        assert err <= (1e-13 if f == "theta" else 1e-14), (f, err)
    assert int(gd["theta_limited_cell_count"]) == wd["theta_limited_cell_count"]
    np.testing.assert_array_equal(gd["theta_first_limited_cell_xyz"].cpu().numpy(), wd["theta_first_limited_cell_xyz"])
    before = wd["theta_mass_before"]
    for k in ("theta_mass_before", "theta_mass_after", "theta_mass_residual"):
        assert abs(float(gd[k]) - wd[k]) <= 1e-12 * max(abs(before), 1.0), k
    if not disable_guards:
        assert wd["theta_limited_cell_count"] == 3
        assert abs(float(gd["theta_mass_residual"])) <= 1e-12 * abs(before)
    del case


def test_epilogue_without_offenders_is_a_noop_for_the_guards(cuda_ready):
    case, origin, cand = _pair(plant=False)
    nl = dycore.OperationalNamelist.from_case(case, run_boundary=False, bc_source="wrfbdy")
    got, gd = dycore.step_epilogue(dycore.State.from_host(cand), dycore.State.from_host(origin), 0.0, nl)
    torch.cuda.synchronize()
    assert int(gd["theta_limited_cell_count"]) == 0
    assert gd["theta_first_limited_cell_xyz"].tolist() == [-1, -1, -1]
    # the limiter is the identity up to the rounding of origin + (candidate -
    # origin) and of the domain sums it redistributes
    assert P.rel_err(got.theta.cpu().numpy(), cand.theta) <= 1e-13
    for f in ("u", "v", "w", "p_total", "ph_total", "mu_total", "qv"):
        np.testing.assert_array_equal(getattr(got, f).cpu().numpy(), getattr(cand, f))
    del case
