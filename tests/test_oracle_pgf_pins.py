"""The oracle's large-step horizontal pressure gradient
(``oracle.dycore.pgf_from_fields`` / ``pgf_dpn``, the terms of
rk_addtend_dry.py:233-362) on the known answers of the reference's own PGF
tests (tests/test_m6x_c2_pgf.py:44-226):

* a horizontally linear hydrostatic set (p = x, pb = 2x, ph' = -8x, al = 3,
  alt = 2) makes the first three terms cancel, in x and in y;
* the fourth (non-hydrostatic) term vanishes without a pressure or dry-mass
  perturbation, and acts with a php gradient and mu' = 25 Pa;
* the surface face of dpn is the cf1/cf2/cf3 extrapolation, the interior
  faces the fnm/fnp interpolation, the top face zero without a lid;
* the map-factor ratio msfux / msfuy and the moisture factor cqu scale the
  final u tendency (msfux doubled and qv = 0.5: ratio 2 / 1.5).

The reference's tests run on its canary grid with flat metrics; the known
answers do not depend on the grid, so a small flat grid is used here."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import dycore as D
from wrf_gpu_b200 import cases

NZ, NY, NX = 8, 10, 12


def _metrics():
    eta = np.linspace(1.0, 0.0, NZ + 1)
    return cases.flat_metrics(eta, NY, NX, 5000.0)


def _fields(**kw):
    z3 = np.zeros((NZ, NY, NX))
    f = dict(ph=np.zeros((NZ + 1, NY, NX)), p=z3.copy(), pb=z3.copy(), al=z3.copy(), alt=np.ones_like(z3),
             mu_total=np.full((NY, NX), 90000.0), mu_pert=np.zeros((NY, NX)))
    f.update(kw)
    ph_tot = f["ph"]  # the base geopotential is zero here
    f["php"] = 0.5 * (ph_tot[:-1] + ph_tot[1:])
    return f


def _pgf(f, m, cqu=None, cqv=None, non_hydrostatic=True):
    ones_u, ones_v = np.ones((NZ, NY, NX + 1)), np.ones((NZ, NY + 1, NX))
    return D.pgf_from_fields(f["ph"], f["p"], f["pb"], f["al"], f["alt"], f["php"], f["mu_total"], f["mu_pert"],
                             ones_u if cqu is None else cqu, ones_v if cqv is None else cqv, m, 1.0 / 3000.0,
                             1.0 / 3000.0, False, non_hydrostatic=non_hydrostatic)


def test_first_three_terms_cancel_in_hydrostatic_balance():
    m = _metrics()
    for axis in (2, 1):
        coord = np.arange(NX if axis == 2 else NY, dtype=np.float64)
        shape = (1, 1, NX) if axis == 2 else (1, NY, 1)
        c = coord.reshape(shape)
        f = _fields(p=np.broadcast_to(c, (NZ, NY, NX)).copy(), pb=np.broadcast_to(2.0 * c, (NZ, NY, NX)).copy(),
                    ph=np.broadcast_to(-8.0 * c, (NZ + 1, NY, NX)).copy(), al=np.full((NZ, NY, NX), 3.0),
                    alt=np.full((NZ, NY, NX), 2.0))
        du, dv = _pgf(f, m, non_hydrostatic=False)
        d = du if axis == 2 else dv
        # interior faces (the edge faces pair a point with itself)
        inner = d[:, :, 1:-1] if axis == 2 else d[:, 1:-1, :]
        assert np.max(np.abs(inner)) < 1.0e-10
        assert np.max(np.abs(d)) < 1.0e-10


def test_fourth_term_vanishes_without_pressure_or_mass_perturbation():
    m = _metrics()
    x = np.arange(NX, dtype=np.float64).reshape(1, 1, NX)
    f = _fields(ph=np.broadcast_to(x, (NZ + 1, NY, NX)).copy(), al=np.zeros((NZ, NY, NX)))
    hyd = _pgf(f, m, non_hydrostatic=False)
    non = _pgf(f, m, non_hydrostatic=True)
    np.testing.assert_allclose(non[0], hyd[0], rtol=1e-12, atol=0.0)
    np.testing.assert_allclose(non[1], hyd[1], rtol=1e-12, atol=0.0)


def test_fourth_term_acts_with_php_gradient_and_mass_perturbation():
    m = _metrics()
    x = np.arange(NX, dtype=np.float64).reshape(1, 1, NX)
    f = _fields(ph=np.broadcast_to(x, (NZ + 1, NY, NX)).copy(), al=np.zeros((NZ, NY, NX)),
                mu_pert=np.full((NY, NX), 25.0), mu_total=np.full((NY, NX), 90025.0))
    hyd = _pgf(f, m, non_hydrostatic=False)
    non = _pgf(f, m, non_hydrostatic=True)
    assert np.max(np.abs(non[0][:, :, 1:-1])) > 0.0
    assert np.max(np.abs((non[0] - hyd[0])[:, :, 1:-1])) > 0.0


def test_dpn_faces_use_cf_surface_and_fnm_fnp_interior_coefficients():
    m = _metrics()
    prof = (np.arange(1, NZ + 1, dtype=np.float64) * 10.0)[:, None, None]
    p = np.broadcast_to(prof, (NZ, NY, NX))
    dpn = D.pgf_dpn(p + p, m, False)  # the pair sum of a horizontally uniform pressure
    bottom = m.cf1 * p[0, 0, 0] + m.cf2 * p[1, 0, 0] + m.cf3 * p[2, 0, 0]
    interior = m.fnm[1] * p[1, 0, 0] + m.fnp[1] * p[0, 0, 0]
    np.testing.assert_allclose(dpn[0], bottom, rtol=1e-14)
    np.testing.assert_allclose(dpn[1], interior, rtol=1e-14)
    assert np.all(dpn[-1] == 0.0)


def test_map_factor_ratio_and_moisture_factor_scale_the_u_tendency():
    m = _metrics()
    ms = SimpleNamespace(**vars(m))
    ms.msfux = m.msfux * 2.0
    x = np.arange(NX, dtype=np.float64).reshape(1, 1, NX)
    f = _fields(ph=np.broadcast_to(x, (NZ + 1, NY, NX)).copy(), al=np.zeros((NZ, NY, NX)))
    dry_du, _ = _pgf(f, m, non_hydrostatic=False)
    zq = np.zeros((NZ, NY, NX))
    moist = SimpleNamespace(qv=np.full((NZ, NY, NX), 0.5), qc=zq, qr=zq, qi=zq, qs=zq, qg=zq)
    cqu, cqv = D.moisture_coupling_factors(moist)
    moist_du, _ = _pgf(f, ms, cqu=cqu, cqv=cqv, non_hydrostatic=False)
    ratio = moist_du[:, :, 1:-1] / dry_du[:, :, 1:-1]
    np.testing.assert_allclose(ratio, 2.0 / 1.5, rtol=1e-12)
