"""The oracle's calc_coef_w (``oracle.dycore.calc_coef_w``, restating
dynamics/acoustic_wrf.py:783-852) on the known answers of the reference's own
top-row regression tests (tests/test_m6b0r_jax_top_row_synthetic.py:114-200,
after WRF's module_small_step_em.F:622-648): the top a row's denominator
takes c1f / c2f at face nz-1, the top b row's at face nz, made distinguishable
by a synthetic profile (c1f = 0.5 and 0 at faces nz-1 and nz, c2f = 1000 and
2000).  With a rigid lid a(nz) = 0 and alpha(nz) = 1 / b_top exactly.  The
expected values use the reference's gravity g = 9.81 (WRF's
module_model_constants value, dynamics/acoustic_wrf.py:53-59); that test file
still writes 9.80665, which the reference's calc_coef_w no longer uses."""

from __future__ import annotations

import numpy as np

from oracle import dycore as D
from wrf_gpu_b200 import cases

G = 9.81


def _metrics(nz=6):
    m = cases.flat_metrics(np.linspace(1.0, 0.0, nz + 1), 1, 1, 5000.0)
    m.c1f = np.asarray(m.c1f, dtype=np.float64).copy()
    m.c2f = np.asarray(m.c2f, dtype=np.float64).copy()
    m.c1f[nz - 1], m.c1f[nz] = 0.5, 0.0
    m.c2f[nz - 1], m.c2f[nz] = 1000.0, 2000.0
    return m


def _coef(m, top_lid, dt=6.0, epssm=0.1):
    nz = m.c1h.shape[0]
    mut = np.array([[90000.0]])
    ones = np.ones((nz + 1, 1, 1))
    c2a = np.ones((nz, 1, 1))
    return D.calc_coef_w(mut, m, dt, epssm, top_lid, ones, c2a), mut, dt, epssm


def test_top_a_row_takes_the_face_below_the_top():
    m = _metrics()
    (a, _, _), mut, dt, epssm = _coef(m, False)
    nz = m.c1h.shape[0]
    cof = (0.5 * dt * G * (1.0 + epssm)) ** 2
    want = -2.0 * cof * m.rdnw[nz - 1] ** 2 / ((m.c1h[nz - 1] * mut + m.c2h[nz - 1]) * (m.c1f[nz - 1] * mut + m.c2f[nz - 1]))
    np.testing.assert_allclose(a[-1], want, rtol=1e-12, atol=0.0)
    assert np.max(np.abs(want)) > 0.0
    wrong = -2.0 * cof * m.rdnw[nz - 1] ** 2 / ((m.c1h[nz - 1] * mut + m.c2h[nz - 1]) * (m.c1f[nz] * mut + m.c2f[nz]))
    assert not np.allclose(wrong, want)  # the profile tells the two faces apart


def test_top_b_row_takes_the_top_face():
    m = _metrics()
    (a, alpha, _), mut, dt, epssm = _coef(m, True)
    nz = m.c1h.shape[0]
    assert np.all(a[-1] == 0.0)
    cof = (0.5 * dt * G * (1.0 + epssm)) ** 2
    b_top = 1.0 + 2.0 * cof * m.rdnw[nz - 1] ** 2 / ((m.c1h[nz - 1] * mut + m.c2h[nz - 1]) * (m.c1f[nz] * mut + m.c2f[nz]))
    np.testing.assert_allclose(1.0 / alpha[-1], b_top, rtol=1e-12, atol=0.0)
