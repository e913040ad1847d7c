"""Oracle pin: rhs_ph's order<=6 specified-boundary branch.

The oracle's vectorised branch (``oracle.dycore.rhs_ph`` with order >= 4 and
specified lateral BCs, core/rhs_ph.py:87-173 and :281-345) is checked against
an explicit per-cell loop restatement of the same row/column rules on the
seeded synthetic fields of the reference's own test of this branch
(tests/test_v014_rhs_ph_real_case.py:26-56: ridge phb, noisy ph/u/v/w/ww,
perturbed map factors, cfn = 1.4, cfn1 = -0.4), at the reference test's
tolerance (atol 1e-7), for a rigid lid and an open top; the WRF gap columns
2 and nx-3 must see no x advection; order 2 stays the periodic operator.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from oracle import dycore as D


def _fields(nz=8, ny=18, nx=20):
    rng = np.random.default_rng(20260611)
    jj, ii = np.mgrid[0:ny, 0:nx]
    ht = 1500.0 * np.exp(-(((ii - nx / 2) / 4.0) ** 2 + ((jj - ny / 2) / 5.0) ** 2))
    lev = np.linspace(0.0, 1.0, nz + 1)[:, None, None]
    f = dict(phb=9.81 * (ht[None] * (1.0 - lev) + 12000.0 * lev))
    f["ph"] = 50.0 * rng.standard_normal((nz + 1, ny, nx))
    f["u"] = 12.0 + 2.0 * rng.standard_normal((nz, ny, nx + 1))
    f["v"] = -6.0 + 2.0 * rng.standard_normal((nz, ny + 1, nx))
    f["w"] = 0.5 * rng.standard_normal((nz + 1, ny, nx))
    ww = 0.2 * rng.standard_normal((nz + 1, ny, nx))
    ww[0] = 0.0
    ww[nz] = 0.0
    f["ww"] = ww
    f["mut"] = 65000.0 + 2000.0 * rng.standard_normal((ny, nx))
    f["muu"] = 65000.0 + 2000.0 * rng.standard_normal((ny, nx + 1))
    f["muv"] = 65000.0 + 2000.0 * rng.standard_normal((ny + 1, nx))
    m = SimpleNamespace(
        c1f=np.linspace(1.0, 0.2, nz + 1), c2f=np.linspace(0.0, 30000.0, nz + 1),
        fnm=np.full(nz, 0.5), fnp=np.full(nz, 0.5), rdnw=np.full(nz, float(nz)),
        msfux=1.0 + 0.02 * rng.standard_normal((ny, nx + 1)),
        msfvy=1.0 + 0.02 * rng.standard_normal((ny + 1, nx)),
        msfty=1.0 + 0.02 * rng.standard_normal((ny, nx)),
        # top-face extrapolation weights 1.4 / -0.4 through the oracle's cfn formula
        dn=np.full(nz, -0.125), dnw=np.full(nz, -0.1))
    return f, m, 1.0 / 3000.0, 1.0 / 3000.0


def _loop_horizontal(f, m, rdx, rdy, top_lid):
    """Per-cell restatement: faces 1..nz-1 use v/u pairs and weight 0.25, the
    open-top face nz uses cfn/cfn1-extrapolated winds and weight 0.5."""
    pht = f["ph"] + f["phb"]
    nz, ny, nx = pht.shape[0] - 1, pht.shape[1], pht.shape[2]
    cfn = (0.5 * m.dnw[-1] + m.dn[-1]) / m.dn[-1]
    cfn1 = -0.5 * m.dnw[-1] / m.dn[-1]
    out = np.zeros_like(pht)
    for k in list(range(1, nz)) + ([] if top_lid else [nz]):
        if k < nz:
            vp, up, wgt = f["v"][k] + f["v"][k - 1], f["u"][k] + f["u"][k - 1], 0.25
        else:
            vp = cfn * f["v"][nz - 1] + cfn1 * f["v"][nz - 2]
            up = cfn * f["u"][nz - 1] + cfn1 * f["u"][nz - 2]
            wgt = 0.5
        fy = (m.c1f[k] * f["muv"] + m.c2f[k]) * vp * m.msfvy
        fx = (m.c1f[k] * f["muu"] + m.c2f[k]) * up * m.msfux
        a = pht[k]
        for j in range(ny):
            for i in range(nx):
                sy = 0.0
                if 3 <= j <= ny - 4:
                    st = (45.0 * (a[j + 1, i] - a[j - 1, i]) - 9.0 * (a[j + 2, i] - a[j - 2, i])
                          + (a[j + 3, i] - a[j - 3, i])) / 60.0
                    sy = (fy[j + 1, i] + fy[j, i]) * st
                elif j in (2, ny - 3):
                    st = (8.0 * (a[j + 1, i] - a[j - 1, i]) - (a[j + 2, i] - a[j - 2, i])) / 12.0
                    sy = (fy[j + 1, i] + fy[j, i]) * st
                elif j in (1, ny - 2):
                    sy = fy[j + 1, i] * (a[j + 1, i] - a[j, i]) + fy[j, i] * (a[j, i] - a[j - 1, i])
                sx = 0.0
                if 3 <= i <= nx - 4:
                    st = (45.0 * (a[j, i + 1] - a[j, i - 1]) - 9.0 * (a[j, i + 2] - a[j, i - 2])
                          + (a[j, i + 3] - a[j, i - 3])) / 60.0
                    sx = (fx[j, i + 1] + fx[j, i]) * st
                elif i in (1, nx - 2):
                    sx = fx[j, i + 1] * (a[j, i + 1] - a[j, i]) + fx[j, i] * (a[j, i] - a[j, i - 1])
                out[k, j, i] -= wgt * rdy / m.msfty[j, i] * sy + wgt * rdx / m.msfty[j, i] * sx
    return out


def _vertical(f, m, top_lid):
    pht = f["ph"] + f["phb"]
    nz = pht.shape[0] - 1
    out = np.zeros_like(pht)
    wdwn = 0.5 * (f["ww"][1:] + f["ww"][:-1]) * m.rdnw[:, None, None] * (pht[1:] - pht[:-1])
    out[1:nz] -= m.fnm[1:nz, None, None] * wdwn[1:nz] + m.fnp[1:nz, None, None] * wdwn[: nz - 1]
    gw = (m.c1f[:, None, None] * f["mut"][None] + m.c2f[:, None, None]) * 9.81 * f["w"] / m.msfty[None]
    out[1:nz] += gw[1:nz]
    out[nz] = 0.0 if top_lid else gw[nz]
    return out


def _oracle(f, m, rdx, rdy, top_lid, order=5, specified=True):
    return D.rhs_ph(f["u"], f["v"], f["ww"], f["ph"], f["phb"], f["w"], f["mut"], f["muu"], f["muv"], m, rdx, rdy,
                    top_lid, order=order, specified=specified)


@pytest.mark.parametrize("top_lid", [True, False])
def test_order6_branch_matches_loop_restatement(top_lid):
    f, m, rdx, rdy = _fields()
    got = _oracle(f, m, rdx, rdy, top_lid)
    want = _vertical(f, m, top_lid) + _loop_horizontal(f, m, rdx, rdy, top_lid)
    np.testing.assert_allclose(got, want, rtol=0.0, atol=1.0e-7)
    assert not top_lid or np.all(got[-1] == 0.0)


def test_order6_gap_columns_have_no_x_advection():
    f, m, rdx, rdy = _fields()
    got = _oracle(f, m, rdx, rdy, True)
    g0 = dict(f, u=np.zeros_like(f["u"]))
    got0 = _oracle(g0, m, rdx, rdy, True)
    nx = f["mut"].shape[1]
    for col in (0, 2, nx - 3, nx - 1):
        np.testing.assert_array_equal(got[:, :, col], got0[:, :, col])
    assert np.abs(got[:, :, 6] - got0[:, :, 6]).max() > 1.0


def test_order2_and_periodic_keep_the_order2_operator():
    f, m, rdx, rdy = _fields()
    ref = D.rhs_ph_order2(f["u"], f["v"], f["ww"], f["ph"], f["phb"], f["w"], f["mut"], f["muu"], f["muv"], m, rdx,
                          rdy, True)
    np.testing.assert_array_equal(_oracle(f, m, rdx, rdy, True, order=2, specified=True), ref)
    np.testing.assert_array_equal(_oracle(f, m, rdx, rdy, True, order=5, specified=False), ref)
