"""Oracle pins: the end-of-step lateral boundary pass
(``apply_lateral_boundaries``, coupling/boundary_apply.py:170-326).

* the reference's own known-answer case (tests/test_m6_boundary_apply.py:
  26-76): uniform boundary strips over a zero interior -- the spec ring takes
  the strip values, the first relax column moves 0.1 of the way (the
  residual Laplacian vanishes for uniform strips), totals are rebuilt from
  the relaxed base and perturbation;
* one field on random data against a per-cell restatement of WRF's
  relax_bdytend value update (W / E columns own rows [b+1, ny-2-b], S / N
  rows own columns [b, nx-1-b], tangential clamp, spec rows last);
* the specified-cadence variant (``dry_spec_only``): ring 0 only, w and p
  untouched, moisture still relaxed.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import dycore as D


def _leaf(value, z, side, width=5, times=2):
    return np.full((times, 4, width, z, side), float(value))


def _kat_state(nx=12, ny=10, nz=4):
    side = max(nx + 1, ny + 1)
    s = SimpleNamespace(
        u=np.zeros((nz, ny, nx + 1)), v=np.zeros((nz, ny + 1, nx)), w=np.zeros((nz + 1, ny, nx)),
        theta=np.zeros((nz, ny, nx)), qv=np.zeros((nz, ny, nx)),
        p_total=np.full((nz, ny, nx), 1000.0), p_perturbation=np.zeros((nz, ny, nx)),
        ph_total=np.full((nz + 1, ny, nx), 100.0), ph_perturbation=np.zeros((nz + 1, ny, nx)),
        mu_total=np.full((ny, nx), 1000.0), mu_perturbation=np.zeros((ny, nx)))
    for q in ("qc", "qr", "qi", "qs", "qg"):
        setattr(s, q, np.zeros((nz, ny, nx)))
    s.theta_bdy, s.qv_bdy = _leaf(10.0, nz, side), _leaf(0.002, nz, side)
    s.u_bdy, s.v_bdy, s.w_bdy = _leaf(3.0, nz, side), _leaf(4.0, nz, side), _leaf(7.0, nz + 1, side)
    s.p_bdy, s.pb_bdy = _leaf(8.0, nz, side), _leaf(900.0, nz, side)
    s.ph_bdy, s.phb_bdy = _leaf(5.0, nz + 1, side), _leaf(95.0, nz + 1, side)
    s.mu_bdy, s.mub_bdy = _leaf(6.0, 1, side), _leaf(990.0, 1, side)
    return s


def _nl(**kw):
    return SimpleNamespace(update_cadence_s=3600.0, spec_zone=1, relax_zone=4, force_geopotential=True, **kw)


def test_reference_known_answer_case():
    out = D.apply_lateral_boundaries(_kat_state(), 0.0, 60.0, _nl())
    assert np.allclose(out.theta[:, 1:-1, 0], 10.0)
    assert np.allclose(out.theta[:, 3:5, 1], 1.0)
    assert np.allclose(out.qv[:, 1:-1, 0], 0.002)
    assert np.all(out.qv >= 0.0)
    assert np.allclose(out.w[:, 1:-1, 0], 7.0)
    assert np.allclose(out.p_perturbation[:, 1:-1, 0], 8.0)
    assert np.allclose(out.p_total[:, 1:-1, 0], 908.0)
    assert np.allclose(out.mu_perturbation[1:-1, 0], 6.0)
    assert np.allclose(out.mu_total[1:-1, 0], 996.0)
    assert np.allclose(out.ph_perturbation[:, 1:-1, 0], 5.0)
    assert np.allclose(out.ph_total[:, 1:-1, 0], 100.0)
    # beyond the relax zone nothing moves
    assert np.all(out.theta[:, 4:-4, 4:-4] == 0.0)


def _literal(field, leaf, dt, lead, cadence):
    """Per-cell WRF relax_bdytend value update, then the spec rows."""
    f = D.interpolate_boundary_leaf(leaf, lead, cadence)
    z, ny, nx = field.shape
    out = field.copy()
    strip = lambda side, b, n: f[side, min(max(b, 0), f.shape[1] - 1), :z, :n]
    for b in (1, 2, 3):
        lin = (5 - (b + 1)) / 3.0
        wf, wg = dt * (0.1 / dt * lin), dt * (1.0 / dt / 50.0 * lin)
        # S / N rows
        for side, row, step in ((2, b, -1), (3, ny - 1 - b, 1)):
            bd = lambda bb: strip(side, bb, nx)
            for i in range(b, nx - b):
                r0 = bd(b)[:, i] - field[:, row, i]
                r1 = bd(b)[:, max(i - 1, 0)] - field[:, row, max(i - 1, 0)]
                r2 = bd(b)[:, min(i + 1, nx - 1)] - field[:, row, min(i + 1, nx - 1)]
                r3 = bd(b - 1)[:, i] - field[:, row + step, i]
                r4 = bd(b + 1)[:, i] - field[:, row - step, i]
                out[:, row, i] = field[:, row, i] + wf * r0 - wg * (r1 + r2 + r3 + r4 - 4.0 * r0)
        # W / E columns
        for side, col, step in ((0, b, -1), (1, nx - 1 - b, 1)):
            bd = lambda bb: strip(side, bb, ny)
            for j in range(b + 1, ny - 1 - b):
                r0 = bd(b)[:, j] - field[:, j, col]
                r1 = bd(b)[:, j - 1] - field[:, j - 1, col]
                r2 = bd(b)[:, j + 1] - field[:, j + 1, col]
                r3 = bd(b - 1)[:, j] - field[:, j, col + step]
                r4 = bd(b + 1)[:, j] - field[:, j, col - step]
                out[:, j, col] = field[:, j, col] + wf * r0 - wg * (r1 + r2 + r3 + r4 - 4.0 * r0)
    out[:, :, 0], out[:, :, nx - 1] = strip(0, 0, ny), strip(1, 0, ny)
    out[:, 0, :], out[:, ny - 1, :] = strip(2, 0, nx), strip(3, 0, nx)
    return out


def test_relax_pass_matches_the_per_cell_stencil():
    rng = np.random.default_rng(4)
    nz, ny, nx = 3, 11, 13
    field = rng.standard_normal((nz, ny, nx))
    leaf = rng.standard_normal((3, 4, 5, nz, max(nx, ny) + 1))
    got = D.lbc_apply_3d(field, leaf, 5400.0, 30.0, 3600.0)
    np.testing.assert_allclose(got, _literal(field, leaf, 30.0, 5400.0, 3600.0), rtol=1e-13, atol=1e-13)


def test_dry_spec_only_pins_ring0_and_leaves_the_rest():
    s = _kat_state()
    rng = np.random.default_rng(2)
    s.theta = rng.standard_normal(s.theta.shape)
    s.w = rng.standard_normal(s.w.shape)
    out = D.apply_lateral_boundaries(s, 0.0, 60.0, _nl(), dry_spec_only=True)
    assert np.allclose(out.theta[:, 0, :], 10.0) and np.allclose(out.theta[:, :, -1], 10.0)
    np.testing.assert_array_equal(out.theta[:, 1:-1, 1:-1], s.theta[:, 1:-1, 1:-1])
    np.testing.assert_array_equal(out.w, s.w)
    np.testing.assert_array_equal(out.p_total, s.p_total)
    assert np.allclose(out.mu_total[0, :], 996.0) and np.allclose(out.ph_total[:, 0, :], 100.0)
    assert np.allclose(out.qv[:, 3:5, 1], 0.0002)  # moisture keeps the full relax pass
