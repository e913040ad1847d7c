"""Oracle pins: the specified-domain boundary cadence (``specified_bdy_cadence``).

Modelled on the reference's own tests of this machinery
(tests/test_v014_specified_bdy_cadence.py): the relax_bdy_dry tendencies
against a literal per-cell restatement of WRF's relax_bdytend stencil (corner
trims, tangential clamps, linear fcx / gcx taper) on seeded fields; the ring-0
theta work pin and the tangential wind work targets against the
small_step_finish reconstruction they are built for; the zero-gradient w work
value against the physical w it must reproduce.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import dycore as D
from tests import parity_util as P
from wrf_gpu_b200 import cases


def _leaf(rng, width, z_len, side_len, scale=1.0, offset=0.0):
    v = rng.normal(size=(1, 4, width, z_len, side_len)) * scale + offset
    return np.repeat(v, 2, axis=0)


def _relax_literal(field, target, dt, spec_zone=1, relax_zone=4):
    """Per-cell WRF relax_bdytend: Y rows own the corners (i in [b, nx-1-b]),
    X columns take rows [b+1, ny-2-b]; tangential neighbours clamped."""
    z, ny, nx = field.shape
    tend = np.zeros_like(field)
    fls = lambda j, i: target[:, j, i] - field[:, j, i]
    for b in range(spec_zone, relax_zone):
        lin = max(0.0, (spec_zone + relax_zone - (b + 1)) / (relax_zone - 1))
        f = 0.1 / dt * lin
        g = 1.0 / dt / 50.0 * lin
        for j, s in ((b, 1), (ny - 1 - b, -1)):
            for i in range(b, nx - b):
                lap = fls(j, max(i - 1, 0)) + fls(j, min(i + 1, nx - 1)) + fls(j - s, i) + fls(j + s, i) - 4.0 * fls(j, i)
                tend[:, j, i] += f * fls(j, i) - g * lap
        for i, s in ((b, 1), (nx - 1 - b, -1)):
            for j in range(b + 1, ny - 1 - b):
                lap = fls(max(j - 1, 0), i) + fls(min(j + 1, ny - 1), i) + fls(j, i - s) + fls(j, i + s) - 4.0 * fls(j, i)
                tend[:, j, i] += f * fls(j, i) - g * lap
    return tend


def _ring(leaf, z, ny, nx):
    out = np.zeros((z, ny, nx))
    for b in range(5):
        out[:, :, b] = leaf[0, b, :z, :ny]
        out[:, :, nx - 1 - b] = leaf[1, b, :z, :ny]
        out[:, b, :] = leaf[2, b, :z, :nx]
        out[:, ny - 1 - b, :] = leaf[3, b, :z, :nx]
    return out


def test_relax_tendencies_match_the_literal_stencil():
    rng = np.random.default_rng(20260611)
    nz, ny, nx, dt = 3, 14, 12, 18.0
    mu_total = 1000.0 + rng.normal(size=(ny, nx))
    side = max(ny + 1, nx + 1)
    ref = SimpleNamespace(
        u=rng.normal(size=(nz, ny, nx + 1)), v=rng.normal(size=(nz, ny + 1, nx)),
        theta=300.0 + rng.normal(size=(nz, ny, nx)), ph_perturbation=10.0 * rng.normal(size=(nz + 1, ny, nx)),
        mu_total=mu_total, mu_perturbation=rng.normal(size=(ny, nx)),
        u_bdy=_leaf(rng, 5, nz, side), v_bdy=_leaf(rng, 5, nz, side), theta_bdy=_leaf(rng, 5, nz, side, 1.0, 300.0),
        ph_bdy=_leaf(rng, 5, nz + 1, side, 10.0), mu_bdy=_leaf(rng, 5, 1, side))
    m = SimpleNamespace(c1h=0.9 + 0.01 * np.arange(nz), c2h=50.0 + np.arange(nz),
                        c1f=0.9 + 0.01 * np.arange(nz + 1), c2f=50.0 + np.arange(nz + 1),
                        msfuy=1.0 + 0.001 * rng.normal(size=(ny, nx + 1)),
                        msfvx=1.0 + 0.001 * rng.normal(size=(ny + 1, nx)),
                        msfty=1.0 + 0.001 * rng.normal(size=(ny, nx)))
    r = D.specified_relax_dry_tendencies(ref, 0.0, m, dt, 3600.0)
    mass_h = m.c1h[:, None, None] * mu_total[None] + m.c2h[:, None, None]
    want_t = _relax_literal(mass_h * ref.theta, mass_h * _ring(ref.theta_bdy[0], nz, ny, nx), dt) / m.msfty[None]
    np.testing.assert_allclose(r.t, want_t, rtol=1e-12, atol=1e-12)
    want_mu = _relax_literal(ref.mu_perturbation[None], _ring(ref.mu_bdy[0], 1, ny, nx), dt)[0]
    np.testing.assert_allclose(r.mu, want_mu, rtol=1e-12, atol=1e-12)
    mass_f = m.c1f[:, None, None] * mu_total[None] + m.c2f[:, None, None]
    want_ph = _relax_literal(mass_f * ref.ph_perturbation, mass_f * _ring(ref.ph_bdy[0], nz + 1, ny, nx), dt) / m.msfty[None]
    np.testing.assert_allclose(r.ph, want_ph, rtol=1e-12, atol=1e-12)
    assert np.all(r.t[:, 0, :] == 0.0) and np.all(r.t[:, 5:-5, 5:-5] == 0.0)
    assert np.abs(r.ru).max() > 0.0 and np.abs(r.rv).max() > 0.0


def test_theta_pin_and_tangential_targets_reconstruct_the_leaves():
    rng = np.random.default_rng(7)
    nz, ny, nx = 3, 8, 9
    c1h, c2h = 0.95 + 0.01 * np.arange(nz), 40.0 + np.arange(nz)
    m = SimpleNamespace(c1h=c1h, c2h=c2h, msfuy=1.0 + 0.001 * rng.normal(size=(ny, nx + 1)),
                        msfvx=1.0 + 0.001 * rng.normal(size=(ny + 1, nx)))
    prep = SimpleNamespace(muu=900.0 + rng.normal(size=(ny, nx + 1)), muus=905.0 + rng.normal(size=(ny, nx + 1)),
                           muv=900.0 + rng.normal(size=(ny + 1, nx)), muvs=905.0 + rng.normal(size=(ny + 1, nx)),
                           u_save=rng.normal(size=(nz, ny, nx + 1)), v_save=rng.normal(size=(nz, ny + 1, nx)))
    side = max(nx + 1, ny + 1)
    ul, vl = _leaf(rng, 5, nz, side, 5.0)[0], _leaf(rng, 5, nz, side, 5.0)[0]
    tu, tv = D.tangential_targets(ul, vl, prep, m)
    mcur = c1h[:, None, None] * prep.muu[None] + c2h[:, None, None]
    mstg = c1h[:, None, None] * prep.muus[None] + c2h[:, None, None]
    for row, s in ((0, 2), (ny - 1, 3)):
        rebuilt = (m.msfuy[row] * tu[:, row, :] + prep.u_save[:, row, :] * mcur[:, row, :]) / mstg[:, row, :]
        np.testing.assert_allclose(rebuilt, ul[s, 0, :nz, :nx + 1], rtol=1e-12)
    vcur = c1h[:, None, None] * prep.muv[None] + c2h[:, None, None]
    vstg = c1h[:, None, None] * prep.muvs[None] + c2h[:, None, None]
    for col, s in ((0, 0), (nx - 1, 1)):
        rebuilt = (m.msfvx[:, col] * tv[:, :, col] + prep.v_save[:, :, col] * vcur[:, :, col]) / vstg[:, :, col]
        np.testing.assert_allclose(rebuilt, vl[s, 0, :nz, :ny + 1], rtol=1e-12)


def test_zero_gradient_w_reproduces_the_interior_physical_w():
    rng = np.random.default_rng(13)
    nzp, ny, nx = 4, 8, 9
    w, w_save = rng.normal(size=(nzp, ny, nx)), 3.0 * rng.normal(size=(nzp, ny, nx))
    mut, muts = 900.0 + rng.normal(size=(ny, nx)), 905.0 + rng.normal(size=(ny, nx))
    m = SimpleNamespace(c1f=0.9 + 0.01 * np.arange(nzp), c2f=30.0 + np.arange(nzp),
                        msfty=1.0 + 0.001 * rng.normal(size=(ny, nx)))
    out = D.specified_w_zero_grad(w, w_save, mut, muts, m)
    mc = m.c1f[:, None, None] * mut[None] + m.c2f[:, None, None]
    ms = m.c1f[:, None, None] * muts[None] + m.c2f[:, None, None]
    before = (m.msfty[None] * w + w_save * mc) / ms
    after = (m.msfty[None] * out + w_save * mc) / ms
    xi = np.clip(np.arange(nx), 1, nx - 2)
    np.testing.assert_allclose(after[:, 0, :], before[:, 1, xi], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(after[:, -1, :], before[:, ny - 2, xi], rtol=1e-12, atol=1e-12)
    yi = np.clip(np.arange(1, ny - 1), 1, ny - 2)
    np.testing.assert_allclose(after[:, 1:-1, 0], before[:, yi, 1], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(after[:, 1:-1, -1], before[:, yi, nx - 2], rtol=1e-12, atol=1e-12)
    np.testing.assert_array_equal(out[:, 1:-1, 1:-1], w[:, 1:-1, 1:-1])


def test_cadence_step_pins_the_ring_to_the_boundary_leaves():
    case = cases.real_like_moist(24, 20, 10, hmax=600.0, specified=True, bdy_noise=True)
    case.controls["specified_bdy_cadence"] = True
    out = P.oracle_steps(case, 1)
    s = out.state
    for f in ("u", "v", "w", "theta", "ph_perturbation", "mu_perturbation"):
        assert np.isfinite(getattr(s, f)).all()
    # the ring-0 theta and mu' land on the leaf values at the step-end lead
    lead = case.controls["dt_s"]
    th_leaf = D.interpolate_boundary_leaf(case.state.theta_bdy, lead, case.controls["update_cadence_s"])
    mu_leaf = D.interpolate_boundary_leaf(case.state.mu_bdy, lead, case.controls["update_cadence_s"])
    nz, ny, nx = s.theta.shape
    np.testing.assert_allclose(s.theta[:, 0, 6:-6], th_leaf[2, 0, :nz, 6:nx - 6], rtol=1e-10)
    np.testing.assert_allclose(s.mu_perturbation[0, 6:-6], mu_leaf[2, 0, 0, 6:nx - 6], rtol=1e-8, atol=1e-8)
    base = cases.real_like_moist(24, 20, 10, hmax=600.0, specified=True, bdy_noise=True)
    ref = P.oracle_steps(base, 1)
    assert np.abs(ref.state.theta - s.theta).max() > 1e-6
