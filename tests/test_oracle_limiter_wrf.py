"""The oracle's positive-definite (opt 1) and monotonic (opt 2) limited scalar
advection (``oracle.dycore.advect_scalar_flux_limited``, restating
flux_advection.py:736-1000) against WRF's own algorithm, restated here as
per-cell loops from ``advect_scalar_pd`` / ``advect_scalar_mono``
(dyn_em/module_advect_em.F):

  1. low-order upwind face fluxes of the old field (Courant-weighted donor
     cell), high-order h5 / v3 face fluxes of the stage field, their
     difference the anti-diffusive flux;
  2. the low-order update of each cell (ph_low), the anti-diffusive mass
     leaving it (flux_out) and, for opt 2, entering it (flux_in) against the
     old field's 7-point extrema;
  3. opt 1: every outgoing anti-diffusive flux of a cell whose outflow
     exceeds its low-order mass is scaled by ph_low / flux_out (each face is
     an outflow of exactly one cell); opt 2: each face flux scaled by the
     smaller of the receiving cell's inflow factor and the donor cell's
     outflow factor;
  4. the tendency from the limited plus low-order fluxes.

The cases are the reference's own parity checks of its limiter against a WRF
transcription (tests/dynamics/test_pd_monotonic_advection.py:387-616): a
top-hat blob carried by a uniform x flow on one periodic row, a column under
a uniform downward-index omega, and a 3-D divergence-free x-z flow, unit map
factors, with the reference's tolerances (1e-13 for the 1-D cases, 1e-12 for
3-D).  The x-z flow here is built from a discrete stream function, so its
flux divergence vanishes exactly.
"""

from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import dycore as D

EPS = 1.0e-20


def _upwind(q_left, q_right, cr):
    a = abs(cr)
    return 0.5 * min(1.0, cr + a) * q_left + 0.5 * max(-1.0, cr - a) * q_right


def _h5(q, vel):
    """WRF flux5 at the face left of q[3] from q[0..5] (i-3 .. i+2), times vel."""
    qm3, qm2, qm1, q0, qp1, qp2 = q
    vel = float(vel)
    f6 = (37.0 * (q0 + qm1) - 8.0 * (qp1 + qm2) + (qp2 + qm3)) / 60.0
    c = ((qp2 - qm3) - 5.0 * (qp1 - qm2) + 10.0 * (q0 - qm1)) / 60.0
    s = (vel > 0.0) - (vel < 0.0)
    return vel * (f6 - s * c)


def _v3(qkm2, qkm1, qk, qkp1, rom):
    """WRF flux3 of the eta-coordinate vertical flux (upwinding on -rom), times rom."""
    rom = float(rom)
    f4 = (7.0 * (qk + qkm1) - (qkp1 + qkm2)) / 12.0
    c = ((qkp1 - qkm2) - 3.0 * (qk - qkm1)) / 12.0
    s = (-rom > 0.0) - (-rom < 0.0)
    return rom * (f4 + s * c)


def wrf_limited_tendency(f, fo, ru, rv, rom, mu, c1, c2, rdx, rdy, rdzw, fzm, fzp, dt, opt, scales=False):
    """advect_scalar_pd (opt 1) / advect_scalar_mono (opt 2), periodic x / y,
    unit map factors; f the stage field, fo the old field, (nz, ny, nx).
    The face masses are the hybrid c1 mu + c2 of the face-averaged column
    mass (x / y) and the average of the two half-level masses (z).  With
    ``scales`` also returns the outflow and inflow factors."""
    nz, ny, nx = f.shape
    dx, dy = 1.0 / rdx, 1.0 / rdy
    mass = lambda k, j, i: c1[k] * mu[j, i] + c2[k]
    # face fluxes: x face (k, j, i) left of cell i, y face below cell j, z face k below level k
    lx = np.zeros((nz, ny, nx)); hx = np.zeros((nz, ny, nx))
    ly = np.zeros((nz, ny, nx)); hy = np.zeros((nz, ny, nx))
    lz = np.zeros((nz + 1, ny, nx)); hz = np.zeros((nz + 1, ny, nx))
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                im1 = (i - 1) % nx
                mu_face = c1[k] * (0.5 * (mu[j, i] + mu[j, im1])) + c2[k]
                lx[k, j, i] = mu_face * (dx / dt) * _upwind(fo[k, j, im1], fo[k, j, i], ru[k, j, i] * dt / dx / mu_face)
                hx[k, j, i] = _h5([f[k, j, (i + d) % nx] for d in range(-3, 3)], ru[k, j, i])
                jm1 = (j - 1) % ny
                mu_face = c1[k] * (0.5 * (mu[j, i] + mu[jm1, i])) + c2[k]
                ly[k, j, i] = mu_face * (dy / dt) * _upwind(fo[k, jm1, i], fo[k, j, i], rv[k, j, i] * dt / dy / mu_face)
                hy[k, j, i] = _h5([f[k, (j + d) % ny, i] for d in range(-3, 3)], rv[k, j, i])
    for k in range(1, nz):
        dz = 2.0 / (rdzw[k] + rdzw[k - 1])
        for j in range(ny):
            for i in range(nx):
                mu_face = 0.5 * (mass(k, j, i) + mass(k - 1, j, i))
                lz[k, j, i] = mu_face * (dz / dt) * _upwind(fo[k - 1, j, i], fo[k, j, i], rom[k, j, i] * dt / dz / mu_face)
                if k == 1 or k == nz - 1:
                    hz[k, j, i] = rom[k, j, i] * (fzm[k] * f[k, j, i] + fzp[k] * f[k - 1, j, i])
                else:
                    hz[k, j, i] = _v3(f[k - 2, j, i], f[k - 1, j, i], f[k, j, i], f[k + 1, j, i], rom[k, j, i])
    ax, ay, az = hx - lx, hy - ly, hz - lz
    s_out = np.ones((nz, ny, nx))
    s_in = np.ones((nz, ny, nx))
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                ip1, jp1 = (i + 1) % nx, (j + 1) % ny
                ph_low = mass(k, j, i) * fo[k, j, i] - dt * (
                    (rdx * (lx[k, j, ip1] - lx[k, j, i]) + rdy * (ly[k, jp1, i] - ly[k, j, i]))
                    + rdzw[k] * (lz[k + 1, j, i] - lz[k, j, i]))
                out = dt * ((rdx * (max(0.0, ax[k, j, ip1]) - min(0.0, ax[k, j, i]))
                             + rdy * (max(0.0, ay[k, jp1, i]) - min(0.0, ay[k, j, i])))
                            + rdzw[k] * (min(0.0, az[k + 1, j, i]) - max(0.0, az[k, j, i])))
                if opt == 1:
                    if out > ph_low:
                        s_out[k, j, i] = max(0.0, ph_low / (out + EPS))
                    continue
                into = -dt * ((rdx * (min(0.0, ax[k, j, ip1]) - max(0.0, ax[k, j, i]))
                               + rdy * (min(0.0, ay[k, jp1, i]) - max(0.0, ay[k, j, i])))
                              + rdzw[k] * (max(0.0, az[k + 1, j, i]) - min(0.0, az[k, j, i])))
                nb = [fo[k, j, i], fo[k, j, (i - 1) % nx], fo[k, j, ip1], fo[k, (j - 1) % ny, i], fo[k, jp1, i],
                      fo[max(k - 1, 0), j, i], fo[min(k + 1, nz - 1), j, i]]
                room_hi = max(nb) * mass(k, j, i) - ph_low
                room_lo = ph_low - min(nb) * mass(k, j, i)
                if into > room_hi:
                    s_in[k, j, i] = max(0.0, room_hi / (into + EPS))
                if out > room_lo:
                    s_out[k, j, i] = max(0.0, room_lo / (out + EPS))
    # limit each anti-diffusive face flux
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                im1, jm1 = (i - 1) % nx, (j - 1) % ny
                for a, donor_pos, recv_pos in ((ax, (k, j, im1), (k, j, i)), (ay, (k, jm1, i), (k, j, i))):
                    v = a[k, j, i]
                    # positive: from the cell below/left (donor) into this cell
                    if opt == 1:
                        a[k, j, i] = s_out[donor_pos] * v if v > 0.0 else (s_out[recv_pos] * v if v < 0.0 else v)
                    else:
                        a[k, j, i] = (min(s_in[recv_pos], s_out[donor_pos]) * v if v > 0.0
                                      else min(s_out[recv_pos], s_in[donor_pos]) * v)
    for k in range(nz + 1):
        below, above = max(k - 1, 0), min(k, nz - 1)
        for j in range(ny):
            for i in range(nx):
                v = az[k, j, i]
                # eta-coordinate face k: a negative flux leaves the cell below it (k-1),
                # a positive one leaves the cell above it (k)
                if opt == 1:
                    az[k, j, i] = s_out[below, j, i] * v if v < 0.0 else (s_out[above, j, i] * v if v > 0.0 else v)
                else:
                    az[k, j, i] = (min(s_in[above, j, i], s_out[below, j, i]) * v if v < 0.0
                                   else min(s_out[above, j, i], s_in[below, j, i]) * v)
    tx, ty, tz = ax + lx, ay + ly, az + lz
    tend = np.zeros((nz, ny, nx))
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                tend[k, j, i] = (-(rdx * (tx[k, j, (i + 1) % nx] - tx[k, j, i]))
                                 - (rdy * (ty[k, (j + 1) % ny, i] - ty[k, j, i]))
                                 - rdzw[k] * (tz[k + 1, j, i] - tz[k, j, i]))
    return (tend, s_out, s_in) if scales else tend


def _oracle(f, fo, ru, rv, rom, mu, c1, c2, rdx, rdy, rdzw, fzm, fzp, dt, opt):
    nz, ny, nx = f.shape
    vel = SimpleNamespace(ru=ru, rv=rv, rom=rom, msftx=np.ones((ny, nx)))
    m = SimpleNamespace(rdnw=rdzw, c1h=c1, c2h=c2, fnm=fzm, fnp=fzp)
    return D.advect_scalar_flux_limited(f, fo, vel, opt, mu, mu, m, rdx, rdy, dt)


def _blob(nz, ny, nx):
    f = np.zeros((nz, ny, nx))
    f[:, ny // 2 - 2: ny // 2 + 2, nx // 2 - 2: nx // 2 + 2] = 1.0
    return f


def _xz_stream_flow(nz, ny, nx, amp):
    """ru (nz, ny, nx) and rom (nz+1, ny, nx) from a stream function on the
    (face, face) corners, zero at the bottom and top faces: the x-z flux
    divergence rdx (ru[i+1] - ru[i]) + rdzw (rom[k+1] - rom[k]) is zero
    exactly for dx = 1 / rdzw = 1."""
    psi = np.zeros((nz + 1, nx + 1))
    for k in range(nz + 1):
        for i in range(nx + 1):
            psi[k, i] = amp * math.sin(2.0 * math.pi * i / nx) * math.sin(math.pi * k / nz)
    psi[:, nx] = psi[:, 0]
    ru = np.empty((nz, ny, nx))
    rom = np.empty((nz + 1, ny, nx))
    for k in range(nz):
        ru[k] = (psi[k + 1, :nx] - psi[k, :nx])[None, :]
    for k in range(nz + 1):
        rom[k] = (-(psi[k, 1:] - psi[k, :nx]))[None, :]
    return ru, rom


def _unit(nz):
    return np.ones(nz), np.zeros(nz), np.ones(nz), np.full(nz, 0.5), np.full(nz, 0.5)


@pytest.mark.parametrize("opt", [1, 2])
def test_limiter_x_row_matches_wrf(opt):
    nz, ny, nx = 4, 1, 24  # identical levels, no vertical flow (the oracle's v3 needs a few levels)
    f = np.zeros((nz, ny, nx))
    f[:, 0, 10:13] = 1.0
    ru = np.full((nz, ny, nx), 1.5)
    rv = np.zeros((nz, ny, nx))
    rom = np.zeros((nz + 1, ny, nx))
    c1, c2, rdzw, fzm, fzp = _unit(nz)
    args = (f, f, ru, rv, rom, np.ones((ny, nx)), c1, c2, 1.0, 1.0, rdzw, fzm, fzp, 0.2, opt)
    want, got = wrf_limited_tendency(*args), _oracle(*args)
    assert np.max(np.abs(got - want)) < 1e-13
    assert np.max(np.abs(want)) > 0.1  # the blob moves


@pytest.mark.parametrize("opt", [1, 2])
def test_limiter_column_matches_wrf(opt):
    nz, ny, nx = 8, 1, 1
    f = np.zeros((nz, ny, nx))
    f[3:5] = 1.0
    ru = np.zeros((nz, ny, nx))
    rv = np.zeros((nz, ny, nx))
    rom = np.zeros((nz + 1, ny, nx))
    rom[1:nz] = 0.05
    c1, c2, rdzw, fzm, fzp = _unit(nz)
    args = (f, f, ru, rv, rom, np.ones((ny, nx)), c1, c2, 1.0, 1.0, rdzw, fzm, fzp, 2.0, opt)
    want, got = wrf_limited_tendency(*args), _oracle(*args)
    assert np.max(np.abs(got - want)) < 1e-13
    assert np.max(np.abs(want)) > 0.01


@pytest.mark.parametrize("opt", [1, 2])
def test_limiter_3d_divergence_free_flow_matches_wrf(opt):
    nz, ny, nx = 8, 8, 24
    f = _blob(nz, ny, nx)
    ru, rom = _xz_stream_flow(nz, ny, nx, 0.3)
    # the flow is exactly non-divergent in x-z
    div = (np.roll(ru, -1, 2) - ru) + (rom[1:] - rom[:nz])
    assert np.max(np.abs(div)) < 1e-15
    rv = np.zeros((nz, ny, nx))
    c1, c2, rdzw, fzm, fzp = _unit(nz)
    args = (f, f, ru, rv, rom, np.ones((ny, nx)), c1, c2, 1.0, 1.0, rdzw, fzm, fzp, 0.5, opt)
    want, s_out, s_in = wrf_limited_tendency(*args, scales=True)
    got = _oracle(*args)
    assert np.max(np.abs(got - want)) < 1e-12
    # the limiter binds (otherwise the case is the plain scheme)
    assert min(s_out.min(), s_in.min()) < 0.5


@pytest.mark.parametrize("opt", [1, 2])
def test_limiter_3d_with_y_flow_and_distinct_old_field(opt):
    """Beyond the reference's cases: a y flow too, an old field that differs
    from the stage field, and a non-uniform column mass with hybrid c1 / c2."""
    rng = np.random.default_rng(3)
    nz, ny, nx = 6, 10, 12
    f = _blob(nz, ny, nx) + 0.05 * rng.random((nz, ny, nx))
    fo = np.clip(f + 0.02 * rng.standard_normal((nz, ny, nx)), 0.0, None)
    ru, rom = _xz_stream_flow(nz, ny, nx, 0.2)
    rv = np.full((nz, ny, nx), -0.4)
    mu = 1.0 + 0.1 * rng.random((ny, nx))
    c1 = np.linspace(1.0, 0.6, nz)
    c2 = np.linspace(0.0, 0.3, nz)
    rdzw = np.full(nz, 1.0)
    fzm, fzp = np.full(nz, 0.5), np.full(nz, 0.5)
    args = (f, fo, ru, rv, rom, mu, c1, c2, 1.0, 1.0, rdzw, fzm, fzp, 0.4, opt)
    want, got = wrf_limited_tendency(*args), _oracle(*args)
    assert np.max(np.abs(got - want)) < 1e-12


@pytest.mark.parametrize("opt", [1, 2])
def test_limited_coupled_tendency_conserves_mass(opt):
    """The reference's moisture-conservation property
    (tests/dynamics/test_moisture_advection_operational.py:153-166): on a
    periodic domain with uniform layers, the coupled limited tendency sums to
    zero relative to the sum of its magnitudes (1e-12)."""
    rng = np.random.default_rng(11)
    nz, ny, nx = 6, 10, 12
    f = _blob(nz, ny, nx) + 0.05 * rng.random((nz, ny, nx))
    fo = np.clip(f + 0.02 * rng.standard_normal((nz, ny, nx)), 0.0, None)
    ru, rom = _xz_stream_flow(nz, ny, nx, 0.25)
    rv = np.full((nz, ny, nx), 0.3)
    mu = 1.0 + 0.1 * rng.random((ny, nx))
    c1, c2, rdzw, fzm, fzp = _unit(nz)
    tend = _oracle(f, fo, ru, rv, rom, mu, c1, c2, 1.0, 1.0, rdzw, fzm, fzp, 0.4, opt)
    assert abs(tend.sum()) / np.abs(tend).sum() < 1e-12
