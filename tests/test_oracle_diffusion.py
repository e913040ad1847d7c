"""Oracle pins: the 6th-order numerical diffusion filter (diff_6th_opt,
dynamics/explicit_diffusion.py:160-226, added in the stage at
runtime/operational_mode.py:2870-2876).

The reference's own tests for it check partition invariance only
(tests/parallel/test_shard_map_dycore.py:51-140), so the restatement is
pinned to known answers of the published stencil (WRF
module_big_step_utilities_em.F:6504-6920, Xue 2000 eq. 3):
* a 2-dx wave f_i = A (-1)^i has fluxes +-32 A (-1)^i, so the filter returns
  -factor / (2 dt) * f per axis (the coefficient factor * 0.015625 / (2 dt)
  times -64);
* a constant field returns zero;
* random fields agree with a per-cell loop of the flux formula with the
  monotonic limiter and wrapped neighbours, for every staggering.
"""

from __future__ import annotations

import numpy as np

from oracle import dycore as D


def test_two_dx_wave_known_answer():
    nz, ny, nx, dt, fac = 3, 6, 8, 6.0, 0.12
    i = np.arange(nx)
    f = np.broadcast_to(2.5 * (-1.0) ** i, (nz, ny, nx)).copy()
    np.testing.assert_allclose(D.sixth_order_diffusion_tendency(f, dt, fac), -fac / (2 * dt) * f, rtol=1e-14)
    j = np.arange(ny)
    g = 2.5 * (-1.0) ** (i[None, None, :] + j[None, :, None]) * np.ones((nz, 1, 1))
    np.testing.assert_allclose(D.sixth_order_diffusion_tendency(g, dt, fac), -2 * fac / (2 * dt) * g, rtol=1e-14)


def test_constant_field_is_untouched():
    f = np.full((4, 5, 7), 300.0)
    assert np.all(D.sixth_order_diffusion_tendency(f, 10.0, 0.12) == 0.0)


def _literal(f, dt, fac):
    coef = fac * 0.015625 / (2.0 * dt)
    nz, ny, nx = f.shape
    out = np.zeros_like(f)

    def axis_term(get, n, m):
        p0 = 10 * (get(m) - get(m - 1)) - 5 * (get(m + 1) - get(m - 2)) + (get(m + 2) - get(m - 3))
        p1 = 10 * (get(m + 1) - get(m)) - 5 * (get(m + 2) - get(m - 1)) + (get(m + 3) - get(m - 2))
        g0, g1 = get(m) - get(m - 1), get(m + 1) - get(m)
        p0 = 0.0 if p0 * g0 <= 0.0 else p0
        p1 = 0.0 if p1 * g1 <= 0.0 else p1
        return coef * (p1 - p0)

    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                t = axis_term(lambda q: f[k, j, q % nx], nx, i)
                if ny > 1:
                    t = t + axis_term(lambda q: f[k, q % ny, i], ny, j)
                out[k, j, i] = t
    return out


def test_random_fields_match_the_per_cell_flux_formula():
    rng = np.random.default_rng(6)
    for shape in ((3, 7, 10), (4, 8, 9), (2, 1, 9), (3, 6, 7)):
        f = 300.0 + rng.standard_normal(shape)
        np.testing.assert_allclose(D.sixth_order_diffusion_tendency(f, 6.0, 0.12), _literal(f, 6.0, 0.12),
                                   rtol=1e-12, atol=1e-13)
