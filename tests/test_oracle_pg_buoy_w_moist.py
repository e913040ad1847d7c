"""The oracle's moist pg_buoy_w (``oracle.dycore.pg_buoy_w_moist``, restating
core/advance_w.py:195-290) on the known answers of the reference's own moist
cqw tests (tests/test_v014_moist_cqw_pressure_dynamics.py:54-96): with no
moisture it is bit-identical to the dry form (the vertical pressure gradient
and buoyancy, and a unit cqw inside / zero at the boundary faces); the
solver's cqw is cq1 = 1 / (1 + the face average of total moisture), strictly
between 0 and 1 for positive moisture; the water loading -cq2 (c1f mub + c2f)
pulls the lower interior faces down.  The reference's synthetic column set."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import dycore as D


def _synthetic():
    rng = np.random.default_rng(7)
    nz, ny, nx = 24, 5, 6
    p = rng.standard_normal((nz, ny, nx)) * 60.0
    mu = rng.standard_normal((ny, nx)) * 40.0
    mub = 1.0e5 + rng.standard_normal((ny, nx)) * 200.0
    m = SimpleNamespace(c1f=np.linspace(1.0, 0.0, nz + 1), c2f=np.linspace(0.0, 1.0, nz + 1),
                        rdn=1.0 / np.linspace(0.02, 0.06, nz), rdnw=1.0 / np.linspace(0.02, 0.06, nz),
                        msfty=1.0 + rng.standard_normal((ny, nx)) * 0.02)
    return nz, ny, nx, p, mu, mub, m


def test_moist_form_without_moisture_is_the_dry_form_bit_for_bit():
    nz, ny, nx, p, mu, mub, m = _synthetic()
    rw_dry, cqw_dry = D.pg_buoy_w_dry(p, mu, m)
    rw_moist, cqw_moist = D.pg_buoy_w_moist(p, mu, mub, np.zeros((nz, ny, nx)), m)
    assert np.array_equal(rw_moist, rw_dry)
    assert np.array_equal(cqw_moist, cqw_dry)
    assert np.all(cqw_dry[1:nz] == 1.0) and np.all(cqw_dry[0] == 0.0) and np.all(cqw_dry[nz] == 0.0)


def test_solver_cqw_is_one_over_one_plus_the_face_moisture():
    rng = np.random.default_rng(3)
    nz, ny, nx, p, mu, mub, m = _synthetic()
    qtot = np.abs(rng.standard_normal((nz, ny, nx))) * 0.01
    _, cqw = D.pg_buoy_w_moist(p, mu, mub, qtot, m)
    face = 0.5 * (qtot[1:nz] + qtot[:nz - 1])
    np.testing.assert_allclose(cqw[1:nz], 1.0 / (1.0 + face), rtol=1e-15)
    assert np.all(cqw[1:nz] < 1.0) and np.all(cqw[1:nz] > 0.0)
    assert np.all(cqw[0] == 0.0) and np.all(cqw[nz] == 0.0)


def test_water_loading_pulls_the_lower_faces_down():
    nz, ny, nx, p, mu, mub, m = _synthetic()
    qtot = np.full((nz, ny, nx), 0.012)
    rw_dry, _ = D.pg_buoy_w_dry(p, mu, m)
    rw_moist, cqw = D.pg_buoy_w_moist(p, mu, mub, qtot, m)
    np.testing.assert_allclose(cqw[1:nz], 1.0 / 1.012, rtol=1e-15)
    assert (rw_moist - rw_dry)[1:6].mean() < 0.0
