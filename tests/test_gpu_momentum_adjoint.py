"""Momentum advection operators and their hand-written adjoints.

``adjoint.advect_u`` / ``adjoint.advect_v`` / ``adjoint.advect_w`` are the
reference's periodic advect_u_flux / advect_v_flux / advect_w_flux
(dynamics/flux_advection.py:1131-1329): the flux-form operator of the CUDA
library (``wrfgpu_flux_advection``) on the core faces, with the transport
velocities averaged to them and the map factors msfux, msfvy (and msfvy /
msfvx on v's vertical term); for w the same operator over w's levels with
the velocities interpolated to them, plus w's own vertical flux divergence
(``wrfgpu_w_vertical_advection``).

* forward: against the oracle's advect_u_flux / advect_v_flux /
  advect_w_flux (rigid lid and open top) on random fields, map factors and
  velocities, 1e-12 relative max-abs;
* adjoint: the operator is bilinear in the advected component and the
  velocities (the upwind switches are fixed by the velocities' signs), so
  with the face-averaged velocities kept away from zero, the directional
  derivatives of <lam, advect(u; ru, rv, rom)> along each input are exact in
  central differences and must equal <grad, d> from the VJP (1e-10), and
  the dot-product identity <L u, lam> = <u, L^T lam> holds to 1e-12.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import dycore as D
from wrf_gpu_b200 import adjoint, cases, dycore

pytestmark = pytest.mark.gpu


def _setup(nx, ny, nz, seed):
    case = cases.warm_bubble_3d(nx, ny, nz)
    rng = np.random.default_rng(seed)
    m = case.metrics
    # non-uniform map factors, so hfac / vfac are exercised
    for n in ("msftx", "msfty", "msfux", "msfuy", "msfvx", "msfvy"):
        a = np.asarray(getattr(m, n))
        setattr(m, n, 1.0 + 0.05 * rng.random(a.shape))
    nl = dycore.OperationalNamelist.from_case(case)
    # velocity magnitudes whose face averages stay away from zero: one sign
    # per field, plus noise smaller than the mean
    ru = 6.0e4 + 1.0e4 * rng.standard_normal((nz, ny, nx))
    rv = -5.0e4 + 1.0e4 * rng.standard_normal((nz, ny, nx))
    rom = 800.0 + 150.0 * rng.standard_normal((nz + 1, ny, nx))
    rom[0] = 0.0
    rom[nz] = 0.0
    u = rng.standard_normal((nz, ny, nx + 1))
    u[..., nx] = u[..., 0]
    v = rng.standard_normal((nz, ny + 1, nx))
    v[:, ny, :] = v[:, 0, :]
    return case, nl, m, u, v, ru, rv, rom, rng


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def _oracle_vel(m, ru, rv, rom, nx, ny):
    return SimpleNamespace(ru=ru, rv=rv, rom=rom, msftx=m.msftx, msfux=np.asarray(m.msfux)[:, :nx],
                           msfvy=np.asarray(m.msfvy)[:ny, :], msfvx=np.asarray(m.msfvx)[:ny, :])


@pytest.mark.parametrize("comp", ["u", "v"])
def test_momentum_advection_matches_oracle(cuda_ready, comp):
    nx, ny, nz = 26, 22, 12
    case, nl, m, u, v, ru, rv, rom, _ = _setup(nx, ny, nz, seed=1)
    vel = _oracle_vel(m, ru, rv, rom, nx, ny)
    rdx, rdy = 1.0 / case.controls["dx"], 1.0 / case.controls["dy"]
    if comp == "u":
        ora = D.advect_u_flux(u, vel, rdx, rdy, m)
        got = adjoint.advect_u(_dev(u), _dev(ru), _dev(rv), _dev(rom), nl)
    else:
        ora = D.advect_v_flux(v, vel, rdx, rdy, m)
        got = adjoint.advect_v(_dev(v), _dev(ru), _dev(rv), _dev(rom), nl)
    got = got.cpu().numpy()
    assert got.shape == ora.shape
    err = np.abs(got - ora).max() / np.abs(ora).max()
    assert err <= 1.0e-12, err


@pytest.mark.parametrize("comp", ["u", "v"])
def test_momentum_advection_vjp(cuda_ready, comp):
    nx, ny, nz = 22, 18, 10
    case, nl, m, u, v, ru, rv, rom, rng = _setup(nx, ny, nz, seed=2)
    op = adjoint.advect_u if comp == "u" else adjoint.advect_v
    f = u if comp == "u" else v
    lam = rng.standard_normal(f.shape)
    LAM = _dev(lam)
    xs = [_dev(a).requires_grad_(True) for a in (f, ru, rv, rom)]
    y = op(*xs, nl)
    grads = torch.autograd.grad(y, xs, grad_outputs=LAM)

    # dot-product identity in the advected component (linear in it)
    lhs = float((y.detach() * LAM).sum())
    rhs = float((grads[0] * xs[0].detach()).sum())
    assert abs(lhs - rhs) <= 1.0e-12 * abs(lhs), (lhs, rhs)

    def inner(*args):
        return float((op(*map(_dev, args), nl) * LAM).sum())

    base = [f, ru, rv, rom]
    # steps small beside the velocities' distance from zero, large enough
    # that rounding stays far below the tolerance
    steps = [1.0, 200.0, 200.0, 5.0]
    for which in range(4):
        d = rng.standard_normal(base[which].shape)
        if which == 3:
            d[0] = 0.0
            d[-1] = 0.0
        if which == 0:  # the wrap face / row does not enter the operator
            if comp == "u":
                d[..., nx] = 0.0
            else:
                d[:, ny, :] = 0.0
        h = steps[which]
        plus = [b.copy() for b in base]
        minus = [b.copy() for b in base]
        plus[which] = plus[which] + h * d
        minus[which] = minus[which] - h * d
        fd = (inner(*plus) - inner(*minus)) / (2 * h)
        ad = float((grads[which] * _dev(d)).sum())
        assert abs(fd - ad) <= 1.0e-10 * max(abs(ad), 1e-300), (comp, which, fd, ad)


@pytest.mark.parametrize("top_lid", [True, False])
def test_w_advection_matches_oracle_and_vjp(cuda_ready, top_lid):
    """advect_w: the horizontal operator on w's levels plus w's vertical flux
    divergence (rigid lid and open top), against the oracle's advect_w_flux
    at 1e-12, and its VJP against central differences along w and each
    velocity (1e-10) with the dot-product identity in w (1e-12)."""
    nx, ny, nz = 24, 20, 12
    case, nl, m, _, _, ru, rv, rom, rng = _setup(nx, ny, nz, seed=4)
    nl.top_lid = top_lid
    w = rng.standard_normal((nz + 1, ny, nx))
    vel = _oracle_vel(m, ru, rv, rom, nx, ny)
    rdx, rdy = 1.0 / case.controls["dx"], 1.0 / case.controls["dy"]
    ora = D.advect_w_flux(w, vel, rdx, rdy, m, top_lid)
    xs = [_dev(a).requires_grad_(True) for a in (w, ru, rv, rom)]
    y = adjoint.advect_w(*xs, nl)
    got = y.detach().cpu().numpy()
    err = np.abs(got - ora).max() / np.abs(ora).max()
    assert err <= 1.0e-12, err

    lam = rng.standard_normal(w.shape)
    LAM = _dev(lam)
    grads = torch.autograd.grad(y, xs, grad_outputs=LAM)
    lhs = float((y.detach() * LAM).sum())
    rhs = float((grads[0] * xs[0].detach()).sum())
    assert abs(lhs - rhs) <= 1.0e-12 * abs(lhs), (lhs, rhs)

    def inner(*args):
        return float((adjoint.advect_w(*map(_dev, args), nl) * LAM).sum())

    base = [w, ru, rv, rom]
    steps = [1.0, 200.0, 200.0, 5.0]
    for which in range(4):
        d = rng.standard_normal(base[which].shape)
        if which == 3:
            d[0] = 0.0
            d[-1] = 0.0
        h = steps[which]
        plus = [b.copy() for b in base]
        minus = [b.copy() for b in base]
        plus[which] = plus[which] + h * d
        minus[which] = minus[which] - h * d
        fd = (inner(*plus) - inner(*minus)) / (2 * h)
        ad = float((grads[which] * _dev(d)).sum())
        assert abs(fd - ad) <= 1.0e-10 * max(abs(ad), 1e-300), (which, fd, ad)
