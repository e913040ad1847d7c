"""Oracle pins: the specified-boundary advection degradation
(``specified_adv_degrade``, flux_advection.py:288-391 and the specified
branches of the scalar / limited / u / v / w operators).

The tiered face fluxes are checked face by face against a literal per-face
restatement of the WRF degrade tiers (the form of the reference's own test,
tests/test_v014_specified_bdy_cadence.py:277-345: seeded field and velocity,
n = 16, with and without the upstream normal-wind rule), the masked
divergence against its definition, and the full-face velocities against the
periodic ones on the faces where both exist.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import dycore as D
from tests import parity_util as P
from wrf_gpu_b200 import cases


def _face_literal(q, vel, m, upstream):
    n = q.shape[0]
    v = vel[m]
    if 3 <= m <= n - 3:
        f6 = (37.0 * (q[m] + q[m - 1]) - 8.0 * (q[m + 1] + q[m - 2]) + (q[m + 2] + q[m - 3])) / 60.0
        c6 = ((q[m + 2] - q[m - 3]) - 5.0 * (q[m + 1] - q[m - 2]) + 10.0 * (q[m] - q[m - 1])) / 60.0
        return v * (f6 - np.sign(v) * c6)
    if m in (2, n - 2):
        f4 = (7.0 * (q[m] + q[m - 1]) - (q[m + 1] + q[m - 2])) / 12.0
        c4 = ((q[m + 1] - q[m - 2]) - 3.0 * (q[m] - q[m - 1])) / 12.0
        return v * (f4 + np.sign(v) * c4)
    if m == 1:
        qb = q[1] if (upstream and q[1] < 0.0) else q[0]
        return v * (0.5 * (q[1] + qb))
    if m == n - 1:
        qb = q[n - 2] if (upstream and q[n - 2] > 0.0) else q[n - 1]
        return v * (0.5 * (q[n - 2] + qb))
    return 0.0


@pytest.mark.parametrize("upstream", [False, True])
@pytest.mark.parametrize("axis", [1, 2])
def test_specified_flux_faces_match_the_tiers(upstream, axis):
    rng = np.random.default_rng(3)
    n = 16
    shape = [2, 3, 3]
    shape[axis] = n
    field = rng.normal(size=shape)
    vel = rng.normal(size=shape)
    got = D.specified_flux_faces(field, vel, axis, upstream=upstream)
    for a in range(shape[0]):
        for b in range(3):
            sl = (a, slice(None), b) if axis == 1 else (a, b, slice(None))
            for m in range(n):
                want = _face_literal(field[sl], vel[sl], m, upstream)
                np.testing.assert_allclose(got[sl][m], want, rtol=1e-13, atol=1e-15)


def test_specified_div_masks_the_outer_cells():
    rng = np.random.default_rng(4)
    fq = rng.normal(size=(2, 3, 12))
    d = D.specified_div(fq, 2)
    assert np.all(d[:, :, 0] == 0.0) and np.all(d[:, :, -1] == 0.0)
    np.testing.assert_array_equal(d[:, :, 1:-1], fq[:, :, 2:] - fq[:, :, 1:-1])


def test_full_face_velocities_equal_periodic_ones_inside():
    case = cases.real_like_moist(24, 20, 6, hmax=600.0, specified=True)
    s, m = case.state, case.metrics
    vel = D.couple_velocities_periodic(s.u, s.v, s.mu_total, m, 1.0 / case.controls["dx"], 1.0 / case.controls["dy"])
    ru_full, rv_full = D.couple_uv_specified(s.u, s.v, s.mu_total, m)
    assert ru_full.shape == s.u.shape and rv_full.shape == s.v.shape
    np.testing.assert_array_equal(ru_full[:, :, 1:24], vel.ru[:, :, 1:24])
    np.testing.assert_array_equal(rv_full[:, 1:20, :], vel.rv[:, 1:20, :])
    assert not np.array_equal(ru_full[:, :, 0], vel.ru[:, :, 0])


def test_degraded_step_runs_and_changes_the_edges():
    case = cases.real_like_moist(24, 20, 8, hmax=600.0, specified=True)
    ref = P.oracle_steps(case, 1)
    case.controls["specified_adv_degrade"] = True
    deg = P.oracle_steps(case, 1)
    for f in ("u", "v", "w", "theta", "qv"):
        assert np.isfinite(getattr(deg.state, f)).all()
    assert np.abs(deg.state.theta - ref.state.theta).max() > 0.0
