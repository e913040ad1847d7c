"""Oracle pins: the RK1-fixed physics tendencies merged into every RK stage
(``rk_addtend_dry``, dynamics/core/rk_addtend_dry.py:490-546, WRF
module_em.F:1711-1786), against the per-field formulas the reference states
(u: (ru_tendf + [rk1] u_save msfuy) / msfuy; v: (rv_tendf + [rk1] v_save
msfvx) * (1/msfvx); w: (rw_tendf + [rk1] w_save msfty) / msfty; theta:
(t_tendf + [rk1] t_save) / msfty + (c1h mut + c2h) h_diabatic / msfty; mu:
+ mu_tendf), and the step with an all-empty bundle equal to the step without
one."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import dycore as D
from tests import parity_util as P
from wrf_gpu_b200 import cases

FIELDS = ("ru_tendf", "rv_tendf", "rw_tendf", "ph_tendf", "t_tendf", "mu_tendf", "h_diabatic", "u_save", "v_save",
          "w_save", "ph_save", "t_save")


def physics_bundle(nz, ny, nx, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    shapes = {"ru_tendf": (nz, ny, nx + 1), "rv_tendf": (nz, ny + 1, nx), "rw_tendf": (nz + 1, ny, nx),
              "ph_tendf": (nz + 1, ny, nx), "t_tendf": (nz, ny, nx), "mu_tendf": (ny, nx), "h_diabatic": (nz, ny, nx),
              "u_save": (nz, ny, nx + 1), "v_save": (nz, ny + 1, nx), "w_save": (nz + 1, ny, nx),
              "ph_save": (nz + 1, ny, nx), "t_save": (nz, ny, nx)}
    mags = {"ru_tendf": 50.0, "rv_tendf": 50.0, "rw_tendf": 20.0, "ph_tendf": 1.0, "t_tendf": 20.0, "mu_tendf": 0.01,
            "h_diabatic": 1.0e-4, "u_save": 1.0e-3, "v_save": 1.0e-3, "w_save": 1.0e-3, "ph_save": 1.0e-2,
            "t_save": 10.0}
    return SimpleNamespace(**{f: scale * mags[f] * rng.standard_normal(shapes[f]) for f in FIELDS})


def test_merge_matches_the_stated_formulas():
    nz, ny, nx = 4, 6, 7
    rng = np.random.default_rng(3)
    m = SimpleNamespace(msfuy=1.0 + 0.01 * rng.random((ny, nx + 1)), msfvx=1.0 + 0.01 * rng.random((ny + 1, nx)),
                        msfty=1.0 + 0.01 * rng.random((ny, nx)), c1h=0.9 + 0.01 * np.arange(nz),
                        c2h=100.0 + np.arange(nz))
    t = SimpleNamespace(u=rng.standard_normal((nz, ny, nx + 1)), v=rng.standard_normal((nz, ny + 1, nx)),
                        w=rng.standard_normal((nz + 1, ny, nx)), theta=rng.standard_normal((nz, ny, nx)),
                        mu=rng.standard_normal((ny, nx)))
    mut = 9.0e4 + rng.standard_normal((ny, nx))
    ph = physics_bundle(nz, ny, nx, 11)
    for rk in (1, 2, 3):
        got = D.rk_addtend_dry(t, ph, rk, m, mut)
        r1 = 1.0 if rk == 1 else 0.0
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    mh = m.c1h[k] * mut[j, i] + m.c2h[k]
                    want = (t.theta[k, j, i] + (ph.t_tendf[k, j, i] + r1 * ph.t_save[k, j, i]) / m.msfty[j, i]
                            + mh * ph.h_diabatic[k, j, i] / m.msfty[j, i])
                    assert abs(got.theta[k, j, i] - want) <= 1e-12 * (abs(want) + 1.0)
        want_u = t.u + (ph.ru_tendf + r1 * ph.u_save * m.msfuy) / m.msfuy
        want_v = t.v + (ph.rv_tendf + r1 * ph.v_save * m.msfvx) / m.msfvx
        want_w = t.w + (ph.rw_tendf + r1 * ph.w_save * m.msfty) / m.msfty
        np.testing.assert_allclose(got.u, want_u, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(got.v, want_v, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(got.w, want_w, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(got.mu, t.mu + ph.mu_tendf, rtol=1e-12, atol=1e-12)


def test_empty_bundle_is_the_plain_step_and_a_full_one_changes_it():
    case = cases.real_like_moist(20, 16, 10, hmax=600.0, specified=True)
    nl = P.oracle_namelist(case)
    empty = SimpleNamespace(**{f: None for f in FIELDS})
    base = P.oracle_steps(case, 1)
    with_empty = P.oracle_steps(case, 1, physics=empty)
    for k in P.STATE_KEYS:
        np.testing.assert_array_equal(getattr(base.state, k), getattr(with_empty.state, k), err_msg=k)
    nz, ny, nx = case.state.theta.shape
    full = P.oracle_steps(case, 1, physics=physics_bundle(nz, ny, nx, 5))
    assert np.abs(full.state.theta - base.state.theta).max() > 1e-6
    assert np.abs(full.state.u - base.state.u).max() > 1e-6
    assert np.isfinite(full.state.w).all()
    del nl
