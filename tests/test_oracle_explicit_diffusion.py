"""The oracle's second-order diffusion closures pinned to known answers.

The known answers are those of the reference's own Smagorinsky tests
(tests/dynamics/test_diffopt1_smagorinsky.py): the deformation of a smooth
periodic flow against its centred differences, zero deformation of a solid
translation, the eddy-viscosity formula with its 10 l cap, zero viscosity
without deformation and xkhh = 3 xkmh, and the flux divergence's zero
domain sum and down-gradient sign.  The constant-K flux form
(explicit_diffusion.py:282-331) is pinned to its discrete Laplacian on a
sine mode and to zero column / domain sums.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import dycore as D


def _analytic_flow(nz=4, ny=24, nx=32, dx=1000.0, dy=1000.0):
    kx, ky = 2.0 * np.pi / (nx * dx), 2.0 * np.pi / (ny * dy)
    xf, xc = np.arange(nx + 1) * dx, (np.arange(nx) + 0.5) * dx
    yf, yc = np.arange(ny + 1) * dy, (np.arange(ny) + 0.5) * dy
    u = np.broadcast_to((np.sin(kx * xf)[None, :] * np.cos(ky * yc)[:, None])[None], (nz, ny, nx + 1)).copy()
    v = np.broadcast_to((np.cos(kx * xc)[None, :] * np.sin(ky * yf)[:, None])[None], (nz, ny + 1, nx)).copy()
    return u, v, dict(kx=kx, ky=ky, xf=xf, xc=xc, yf=yf, yc=yc, dx=dx, dy=dy, nz=nz, ny=ny, nx=nx)


def test_deformation_of_a_smooth_flow():
    u, v, a = _analytic_flow()
    d11, d22, d12 = D.horizontal_deformation_2d(u, v, a["dx"], a["dy"])
    kx, ky, xf, xc, yf, yc = a["kx"], a["ky"], a["xf"], a["xc"], a["yf"], a["yc"]
    want11 = 2.0 * (np.sin(kx * xf[1:]) - np.sin(kx * xf[:-1]))[None, :] / a["dx"] * np.cos(ky * yc)[:, None]
    want22 = 2.0 * np.cos(kx * xc)[None, :] * (np.sin(ky * yf[1:]) - np.sin(ky * yf[:-1]))[:, None] / a["dy"]
    np.testing.assert_allclose(d11, np.broadcast_to(want11, d11.shape), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(d22, np.broadcast_to(want22, d22.shape), rtol=1e-12, atol=1e-12)
    # D12 on the SW corner: (u(j) - u(j-1)) / dy + (v(i) - v(i-1)) / dx, periodic
    um, vm = u[:, :, :-1], v[:, :-1, :]
    want12 = (um - np.roll(um, 1, 1)) / a["dy"] + (vm - np.roll(vm, 1, 2)) / a["dx"]
    np.testing.assert_allclose(d12, want12, rtol=1e-12, atol=1e-12)


def test_solid_translation_has_no_deformation():
    nz, ny, nx = 3, 16, 20
    d11, d22, d12 = D.horizontal_deformation_2d(np.full((nz, ny, nx + 1), 5.0), np.full((nz, ny + 1, nx), -3.0),
                                                500.0, 500.0)
    for d in (d11, d22, d12):
        assert np.all(d == 0.0)


def test_eddy_viscosity_formula_cap_and_zero():
    rng = np.random.default_rng(0)
    nz, ny, nx, dx, dy = 4, 18, 22, 750.0, 750.0
    d11, d22, d12 = (1e-4 * rng.standard_normal((nz, ny, nx)) for _ in range(3))
    km, kh = D.smag2d_horizontal_km(d11, d22, d12, dx, dy, 0.25)
    tmp = 0.25 * (d12 + np.roll(d12, -1, 1) + np.roll(d12, -1, 2) + np.roll(np.roll(d12, -1, 1), -1, 2))
    want = 0.25 ** 2 * dx * dy * np.sqrt(0.25 * (d11 - d22) ** 2 + tmp ** 2)
    np.testing.assert_allclose(km, want, rtol=1e-12)
    np.testing.assert_allclose(kh, 3.0 * km, rtol=1e-12)
    big = np.ones((2, 8, 8))
    km_big, _ = D.smag2d_horizontal_km(big, 0.0 * big, 0.0 * big, 1000.0, 1000.0, 0.25)
    np.testing.assert_allclose(km_big, 10.0 * 1000.0, rtol=1e-12)  # the 10 l ceiling
    z = np.zeros((3, 8, 8))
    km0, kh0 = D.smag2d_horizontal_km(z, z, z, 1000.0, 1000.0, 0.25)
    assert np.all(km0 == 0.0) and np.all(kh0 == 0.0)


def test_flux_divergence_conserves_and_diffuses_down_gradient():
    rng = np.random.default_rng(2)
    nz, ny, nx = 4, 16, 18
    field = 300.0 + rng.standard_normal((nz, ny, nx))
    k = 60.0 + 20.0 * rng.random((nz, ny, nx))
    mass = 9.0e4 + 1.0e3 * rng.standard_normal((nz, ny, nx))
    tend = D.hdiff_coord(field, k, mass, 1000.0, 1000.0)
    assert np.max(np.abs(tend.sum(axis=(1, 2)))) < 1e-6 * np.abs(tend).max() * nx * ny
    nx = 32
    xc = (np.arange(nx) + 0.5) * 500.0
    f = np.broadcast_to(np.sin(2.0 * np.pi * xc / (nx * 500.0))[None, None, :], (4, 1, nx)).copy()
    t = D.hdiff_coord(f, np.full(f.shape, 75.0), np.full(f.shape, 9.0e4), 500.0, 500.0)
    assert np.sum(t[0, 0] * f[0, 0]) < 0.0


def test_smagorinsky_tendencies_vanish_for_a_uniform_state():
    nz, ny, nx = 5, 7, 9
    s = SimpleNamespace(u=np.full((nz, ny, nx + 1), 7.0), v=np.full((nz, ny + 1, nx), -2.0),
                        w=np.full((nz + 1, ny, nx), 0.3), theta=np.full((nz, ny, nx), 301.0))
    ones = lambda *sh: np.full(sh, 9.0e4)
    out = D.smagorinsky_2d_tendencies(s, ones(nz, ny, nx + 1), ones(nz, ny + 1, nx), ones(nz, ny, nx),
                                      ones(nz + 1, ny, nx), 1000.0, 1000.0, 0.25)
    for t in out:
        assert np.all(t == 0.0)
    assert out[0].shape == (nz, ny, nx + 1) and out[1].shape == (nz, ny + 1, nx) and out[2].shape == (nz + 1, ny, nx)


def test_constant_k_flux_form_on_a_sine_mode():
    nz, ny, nx, dx, dy, dz = 6, 10, 16, 800.0, 900.0, 300.0
    kx = 2.0 * np.pi / nx
    xc = np.arange(nx)
    f = np.broadcast_to(np.sin(kx * xc)[None, None, :], (nz, ny, nx)).copy()
    mass, nu = np.full(f.shape, 9.0e4), 75.0
    t = D.const_k_diffusion(f, mass, nu, dx, dy, dz)
    lap = -4.0 * np.sin(kx / 2.0) ** 2 / dx ** 2  # the discrete Laplacian's eigenvalue
    np.testing.assert_allclose(t, mass * nu * lap * f, rtol=1e-10, atol=1e-12 * np.abs(t).max())
    rng = np.random.default_rng(4)
    g = rng.standard_normal((nz, ny, nx))
    m = 9.0e4 + 1.0e3 * rng.standard_normal((nz, ny, nx))
    tg = D.const_k_diffusion(g, m, nu, dx, dy, dz)
    # zero-flux top / bottom and periodic sides: the domain sum vanishes
    assert abs(tg.sum()) < 1e-9 * np.abs(tg).sum()
    assert D.const_k_dz(np.cumsum(np.full((nz + 1, ny, nx), 9.81 * 400.0), axis=0)) == 400.0
