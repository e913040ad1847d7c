"""Oracle pins: the post-step guards (runtime/operational_mode.py:1300-1520)
and their order around the end-of-step boundary pass (:4950-4983).

* the reference's limiter known-answer cases (tests/savepoint/
  test_dycore_limiter.py:9-59): two offending cells clipped into [0, 1000] K,
  counted, the first reported as [x, y, z] = [1, 0, 0], the mass integral
  kept; a no-op candidate passes through with the empty record; per-cell
  monotonic bounds honoured;
* the reference's dry-mass guard case (tests/test_m7_skill_fix_algorithmic.py:
  105-115): a negative mu falls back to the origin;
* the mixing-ratio and finite guards, and the epilogue's order: guards before
  the boundary pass see the raw step output, guards after it the bounded one.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import dycore as D
from tests import parity_util as P


def test_limiter_clips_counts_first_cell_and_conserves_mass():
    origin = np.full((1, 2, 3), 300.0)
    cand = origin.copy()
    cand[0, 0, 1], cand[0, 1, 2] = -10.0, 1110.0
    lim, d = D.theta_increment_limiter(cand, origin, np.ones_like(origin))
    assert lim.min() >= 0.0 and lim.max() <= 1000.0
    assert d["theta_limited_cell_count"] == 2
    np.testing.assert_array_equal(d["theta_first_limited_cell_xyz"], [1, 0, 0])
    assert abs(d["theta_mass_residual"]) < 1e-9
    assert abs(d["theta_mass_before"] - d["theta_mass_after"]) < 1e-9


def test_limiter_noop_records_empty_diagnostics():
    origin = np.full((1, 2, 3), 300.0)
    lim, d = D.theta_increment_limiter(origin + 2.0, origin, np.ones_like(origin))
    np.testing.assert_allclose(lim, origin + 2.0)
    assert d["theta_limited_cell_count"] == 0
    np.testing.assert_array_equal(d["theta_first_limited_cell_xyz"], [-1, -1, -1])
    assert abs(d["theta_mass_residual"]) < 1e-9


def test_limiter_honours_monotonic_bounds():
    origin = np.array([[[290.0, 300.0, 310.0]]])
    cand = origin.copy()
    cand[0, 0, 1] = 100.0
    lim, d = D.theta_increment_limiter(cand, origin, np.ones_like(origin),
                                       lower_bound=np.array([[[290.0, 290.0, 300.0]]]),
                                       upper_bound=np.array([[[300.0, 310.0, 310.0]]]))
    assert lim[0, 0, 1] >= 290.0
    assert d["theta_limited_cell_count"] == 1
    np.testing.assert_array_equal(d["theta_first_limited_cell_xyz"], [1, 0, 0])


def test_limiter_replaces_non_finite_and_weights_by_mass():
    rng = np.random.default_rng(3)
    origin = 300.0 + rng.standard_normal((3, 4, 5))
    cand = origin + rng.standard_normal(origin.shape)
    cand[1, 2, 3], cand[2, 0, 0], cand[0, 3, 1] = np.nan, np.inf, 1500.0
    mass = np.broadcast_to(rng.uniform(5e3, 9e4, (4, 5))[None], origin.shape)
    lim, d = D.theta_increment_limiter(cand, origin, mass)
    assert np.all(np.isfinite(lim)) and lim.max() <= 1000.0
    assert d["theta_limited_cell_count"] == 3
    np.testing.assert_array_equal(d["theta_first_limited_cell_xyz"], [1, 3, 0])
    # the clipped increments are spread over the domain: the integral is kept
    fc = np.where(np.isfinite(cand), cand, origin)
    assert abs(np.sum(lim * mass) - np.sum(fc * mass)) <= 1e-12 * np.sum(fc * mass)


def test_mass_guard_restores_negative_mu():
    origin = SimpleNamespace(mu_total=np.full((3, 4), 9e4), mu_perturbation=np.full((3, 4), 10.0))
    bad = SimpleNamespace(mu_total=np.full((3, 4), -5.0), mu_perturbation=np.full((3, 4), -5.0))
    g = D.limit_guarded_mass_state(bad, origin)
    assert g.mu_total.min() >= 1.0
    np.testing.assert_array_equal(g.mu_perturbation, origin.mu_perturbation)


def test_mixing_ratio_and_finite_guards():
    o = np.full(6, 1e-3)
    c = np.array([2e-3, -1e-9, 0.06, np.nan, np.inf, 0.05])
    np.testing.assert_array_equal(D.valid_mixing_ratio(c, o), [2e-3, 1e-3, 1e-3, 1e-3, 1e-3, 0.05])
    np.testing.assert_array_equal(D.finite_or_origin(c, o), [2e-3, -1e-9, 0.06, 1e-3, 1e-3, 0.05])


def _pair():
    from wrf_gpu_b200 import cases
    case = cases.real_like_moist(20, 16, 6, hmax=600.0, specified=True, bdy_noise=True)
    origin = D.copy_state(case.state)
    cand = D.copy_state(origin)
    rng = np.random.default_rng(5)
    P.attach_lbc_leaves(origin, rng)
    cand = D.copy_state(origin)
    cand.theta = cand.theta + rng.standard_normal(cand.theta.shape)
    cand.theta[2, 1, 1], cand.theta[3, 8, 9] = np.nan, 1200.0      # one on the ring, one inside
    cand.qv[1, 8, 8], cand.qc[0, 0, 0] = 0.2, -1.0
    cand.mu_perturbation[7, 7], cand.mu_total[7, 7] = np.nan, np.nan
    cand.u[0, 8, 8] = np.inf
    return case, origin, cand


def test_epilogue_orders_guards_around_the_boundary_pass():
    case, origin, cand = _pair()
    nl = SimpleNamespace(update_cadence_s=3600.0, spec_zone=1, relax_zone=4, force_geopotential=True)
    s, d = D.step_epilogue(cand, origin, 1800.0, 6.0, nl, run_boundary=True)
    assert d["theta_limited_cell_count"] == 2
    np.testing.assert_array_equal(d["theta_first_limited_cell_xyz"], [1, 1, 2])
    assert s.qv[1, 8, 8] == origin.qv[1, 8, 8] and s.qc[0, 0, 0] >= 0.0
    assert s.mu_total[7, 7] == origin.mu_total[7, 7]
    assert s.u[0, 8, 8] == origin.u[0, 8, 8]
    for f in ("u", "v", "w", "theta", "p_total", "ph_total", "mu_total", "qv"):
        assert np.all(np.isfinite(getattr(s, f))), f
    # guards off: the boundary pass alone
    s2, d2 = D.step_epilogue(cand, origin, 1800.0, 6.0, nl, run_boundary=True, disable_guards=True)
    assert d2["theta_limited_cell_count"] == 0
    want = D.apply_lateral_boundaries(cand, 1800.0, 6.0, nl)
    np.testing.assert_array_equal(s2.theta, want.theta)
    # no boundary: the dynamics guards only, the winds untouched
    s3, _ = D.step_epilogue(cand, origin, 1800.0, 6.0, nl, run_boundary=False)
    assert np.isinf(s3.u[0, 8, 8])
    del case
