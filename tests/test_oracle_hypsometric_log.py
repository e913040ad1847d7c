"""The oracle's hypsometric_opt = 2 (log-pressure) diagnostics
(``oracle.dycore.absolute_diagnostics`` / ``_log_alpha``, restating
rk_addtend_dry.py:127-230) on the analytic known answer of the reference's
own regression test (tests/test_v014_hypsometric_opt2.py:38-112): a column
integrated from a known total specific volume alpha_t with the exact log
relation ph(k+1) = ph(k) + alpha_t(k) phm(k) log(pfd(k) / pfu(k)) is inverted
exactly (1e-12), the perturbation al is alpha_t minus the log-form base
(1e-10), and the linear (hypsometric_opt = 1) form shows its one-signed
O((dp/p)^2) deviation.  The base state is the 3-D warm bubble's."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import dycore as D
from wrf_gpu_b200 import cases


def _column():
    case = cases.warm_bubble_3d(16, 12, 20)
    s, m = case.state, case.metrics
    col = lambda a: np.asarray(a, dtype=np.float64)[:, None, None]
    mub = s.mu_total - s.mu_perturbation
    phb = s.ph_total - s.ph_perturbation
    nz, ny, nx = s.theta.shape
    rng = np.random.default_rng(20260611)
    mu_pert = 50.0 * (1.0 + 0.1 * rng.standard_normal((ny, nx)))
    muts = mub + mu_pert
    alb = -(phb[1:] - phb[:-1]) / (col(m.dnw) * (col(m.c1h) * mub[None] + col(m.c2h)))
    alpha_t = alb * (1.0 + 0.02 * np.sin(np.linspace(0.0, 3.0, nz))[:, None, None])
    p_top = float(m.p_top)
    pfu = col(m.c3f[1:]) * muts[None] + col(m.c4f[1:]) + p_top
    pfd = col(m.c3f[:-1]) * muts[None] + col(m.c4f[:-1]) + p_top
    phm = col(m.c3h) * muts[None] + col(m.c4h) + p_top
    ph_tot = np.zeros((nz + 1, ny, nx))
    ph_tot[0] = phb[0]
    for k in range(nz):
        ph_tot[k + 1] = ph_tot[k] + alpha_t[k] * phm[k] * np.log(pfd[k] / pfu[k])
    st = SimpleNamespace(**vars(s))
    st.ph_total, st.ph_perturbation = ph_tot, ph_tot - phb
    st.mu_total, st.mu_perturbation = mub + mu_pert, mu_pert
    return st, m, alpha_t, alb, mub, phb, muts


def test_log_form_inverts_the_log_column_exactly():
    st, m, alpha_t, alb, mub, phb, muts = _column()
    dph = st.ph_total[1:] - st.ph_total[:-1]
    alt_log = D._log_alpha(dph, muts[None], m)
    assert np.max(np.abs(alt_log - alpha_t) / np.abs(alpha_t)) < 1e-12
    _, _, al2, _, _ = D.absolute_diagnostics(st, m, 2)
    alb_log = D._log_alpha(phb[1:] - phb[:-1], mub[None], m)
    np.testing.assert_allclose(al2, alpha_t - alb_log, rtol=0.0, atol=1e-10)


def test_linear_form_deviates_one_signed():
    st, m, alpha_t, alb, mub, phb, muts = _column()
    _, _, al1, _, _ = D.absolute_diagnostics(st, m, 1)
    alt1 = al1 + alb  # the linear form's total: perturbation plus the linear base
    dph = st.ph_total[1:] - st.ph_total[:-1]
    alt2 = D._log_alpha(dph, muts[None], m)
    assert np.max(np.abs(alt1 - alpha_t) / np.abs(alpha_t)) > 1e-7
    assert np.min(alt1 - alt2) > 0.0
