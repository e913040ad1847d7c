"""The oracle's vertical flux divergence of w (``oracle.dycore._vdiv_w``,
flux_advection.py's w advection) at the model top, on the known answers of
the reference's own top-face tests (tests/dynamics/test_advect_w_topface.py:
42-87, after WRF's advect_w, module_advect_em.F vert_order 3): with a rigid
lid the top face's tendency is zero; with an open top it is the lid pickup
2 rdn(nz-1) vflux(nz), vflux(nz) = 0.5 (rom(nz) + rom(nz-1)) 0.5 (w(nz) +
w(nz-1)); the top flux enters the divergence of face nz-1 and no face below
it.  Seeded random columns, as in the reference's tests."""

from __future__ import annotations

import numpy as np

from oracle import dycore as D


def _column(seed, nz=12, nx=16):
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((nz + 1, 1, nx))
    rom = rng.standard_normal((nz + 1, 1, nx))
    rdn = rng.uniform(0.8, 1.2, size=nz)
    return w, rom, rdn


def test_rigid_lid_top_face_tendency_is_zero():
    w, rom, rdn = _column(1)
    tend = D._vdiv_w(w, rom, rdn, True)
    assert np.all(tend[-1] == 0.0)


def test_open_top_face_tendency_is_the_lid_pickup():
    w, rom, rdn = _column(2)
    nz = rdn.size
    tend = D._vdiv_w(w, rom, rdn, False)
    vflux_top = 0.5 * (rom[nz] + rom[nz - 1]) * 0.5 * (w[nz] + w[nz - 1])
    np.testing.assert_allclose(tend[nz], 2.0 * rdn[nz - 1] * vflux_top, rtol=1e-13, atol=1e-15)
    assert np.max(np.abs(tend[nz])) > 0.0


def test_open_top_flux_enters_face_nz_minus_1_only():
    w, rom, rdn = _column(3)
    nz = rdn.size
    lid = D._vdiv_w(w, rom, rdn, True)
    open_ = D._vdiv_w(w, rom, rdn, False)
    assert np.all(open_[1:nz - 1] == lid[1:nz - 1])
    assert np.max(np.abs(open_[nz - 1] - lid[nz - 1])) > 0.0
