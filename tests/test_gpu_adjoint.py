"""The hand-written adjoint of the flux-form scalar advection operator.

* forward: the CUDA operator against the oracle's advect_scalar_flux
  (flux_advection.py:482-568) on random fields and velocities, 1e-12;
* adjoint: the dot-product identity <L q, lam> = <q, L^T lam> to 1e-12
  relative, and central finite differences of J(q) = 0.5 |L q|^2 along random
  directions against <grad J, d> from torch autograd (1e-8: the operator is
  linear, so the differences are exact up to rounding);
* velocity adjoint: the operator is bilinear in q and the transport
  velocities (the upwind switches fixed by the velocities' signs), so with
  the velocities kept away from zero the directional derivative of
  <lam, L(ru, rv, rom) q> along (d ru, d rv, d rom) is exact in central
  differences; it must equal <ru_bar, d ru> + <rv_bar, d rv> + <rom_bar, d rom>
  (1e-10), field by field and through torch autograd together with q;
* cost: the adjoint launch against the forward launch at 433 x 433 x 50
  (the stated bound is 3x).
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import dycore as D
from wrf_gpu_b200 import adjoint, cases, dycore

pytestmark = pytest.mark.gpu


def _setup(nx, ny, nz, seed=0):
    case = cases.warm_bubble_3d(nx, ny, nz)
    nl = dycore.OperationalNamelist.from_case(case)
    rng = np.random.default_rng(seed)
    q = rng.standard_normal((nz, ny, nx))
    ru = 5.0e4 * rng.standard_normal((nz, ny, nx))
    rv = 5.0e4 * rng.standard_normal((nz, ny, nx))
    rom = 1.0e3 * rng.standard_normal((nz + 1, ny, nx))
    rom[0] = 0.0
    rom[nz] = 0.0
    dev = lambda a: torch.as_tensor(a, device="cuda")
    return case, nl, q, ru, rv, rom, dev


def test_forward_operator_matches_oracle(cuda_ready):
    case, nl, q, ru, rv, rom, dev = _setup(24, 20, 12)
    m = case.metrics
    vel = SimpleNamespace(ru=ru, rv=rv, rom=rom, msftx=m.msftx)
    ora = D.advect_scalar_flux(q, vel, 1.0 / case.controls["dx"], 1.0 / case.controls["dy"], m.rdnw, m.fnm, m.fnp)
    got = adjoint.scalar_advection(dev(q), dev(ru), dev(rv), dev(rom), nl).cpu().numpy()
    err = np.abs(got - ora).max() / np.abs(ora).max()
    assert err <= 1.0e-12, err


def test_adjoint_dot_product_and_finite_differences(cuda_ready):
    case, nl, q, ru, rv, rom, dev = _setup(20, 18, 10, seed=1)
    rng = np.random.default_rng(2)
    lam = dev(rng.standard_normal(q.shape))
    qd = dev(q).requires_grad_(True)
    Lq = adjoint.scalar_advection(qd, dev(ru), dev(rv), dev(rom), nl)
    (qbar,) = torch.autograd.grad(Lq, qd, grad_outputs=lam)
    lhs = float((Lq.detach() * lam).sum())
    rhs = float((dev(q) * qbar).sum())
    assert abs(lhs - rhs) / max(abs(lhs), 1e-300) <= 1.0e-12, (lhs, rhs)

    def J(x):
        y = adjoint.scalar_advection(x, dev(ru), dev(rv), dev(rom), nl)
        return 0.5 * (y * y).sum()

    qd = dev(q).requires_grad_(True)
    (g,) = torch.autograd.grad(J(qd), qd)
    for n in range(8):
        d = dev(np.random.default_rng(10 + n).standard_normal(q.shape))
        h = 1.0e-3
        fd = (float(J(dev(q) + h * d)) - float(J(dev(q) - h * d))) / (2 * h)
        ad = float((g * d).sum())
        assert abs(fd - ad) / abs(ad) <= 1.0e-8, (n, fd, ad)


def test_adjoint_cost_relative_to_forward(cuda_ready):
    case, nl, q, ru, rv, rom, dev = _setup(433, 433, 50, seed=3)
    op = adjoint._Op(nl)
    Q, RU, RV, ROM = dev(q), dev(ru), dev(rv), dev(rom)
    out = torch.empty_like(Q)

    def timed(name, src):
        for _ in range(3):
            op.apply(name, src, RU, RV, ROM, out)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            op.apply(name, src, RU, RV, ROM, out)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 10

    t_fwd = timed("wrfgpu_scalar_advection", Q)
    t_adj = timed("wrfgpu_scalar_advection_adjoint", Q)
    print(f"scalar advection at 433x433x50: forward {t_fwd:.3f} ms, adjoint {t_adj:.3f} ms, ratio {t_adj / t_fwd:.2f}")
    assert t_adj <= 3.0 * t_fwd


def _away_from_zero(a, floor):
    """The same random field with every magnitude at least ``floor``, so a
    small perturbation never flips an upwind switch."""
    return np.where(a >= 0.0, a + floor, a - floor)


def test_velocity_adjoint_matches_directional_derivatives(cuda_ready):
    case, nl, q, ru, rv, rom, dev = _setup(22, 18, 12, seed=5)
    ru, rv = _away_from_zero(ru, 1.0e3), _away_from_zero(rv, 1.0e3)
    rom = rom.copy()
    rom[1:-1] = _away_from_zero(rom[1:-1], 50.0)
    rng = np.random.default_rng(6)
    lam = rng.standard_normal(q.shape)
    Q, LAM = dev(q), dev(lam)
    vel = [dev(ru).requires_grad_(True), dev(rv).requires_grad_(True), dev(rom).requires_grad_(True)]
    Lq = adjoint.scalar_advection(Q, *vel, nl)
    bars = torch.autograd.grad(Lq, vel, grad_outputs=LAM)
    assert float(bars[2][0].abs().max()) == 0.0 and float(bars[2][-1].abs().max()) == 0.0

    def inner(ru_, rv_, rom_):
        return float((adjoint.scalar_advection(Q, dev(ru_), dev(rv_), dev(rom_), nl) * LAM).sum())

    base = (ru, rv, rom)
    for which in range(3):
        d = rng.standard_normal(base[which].shape)
        if which == 2:
            d[0] = 0.0
            d[-1] = 0.0
        # steps well below the velocity floors (10 and 20 standard
        # deviations), large enough that the rounding of the two inner
        # products stays far below the tolerance
        h = 5.0 if which == 2 else 100.0
        plus = [b.copy() for b in base]
        minus = [b.copy() for b in base]
        plus[which] = plus[which] + h * d
        minus[which] = minus[which] - h * d
        fd = (inner(*plus) - inner(*minus)) / (2 * h)
        ad = float((bars[which] * dev(d)).sum())
        assert abs(fd - ad) <= 1.0e-10 * max(abs(ad), 1e-300), (which, fd, ad)


def test_velocity_and_field_gradients_together(cuda_ready):
    """J = 0.5 |L(ru, rv, rom) q|^2 differentiated with respect to q and all
    three velocities at once, against central differences along a joint
    random direction (J is a polynomial of degree 4 there: the central
    difference error is O(h^2), bounded by the 1e-7 tolerance at h = 1e-4)."""
    case, nl, q, ru, rv, rom, dev = _setup(20, 16, 10, seed=8)
    ru, rv = _away_from_zero(ru, 1.0e3), _away_from_zero(rv, 1.0e3)
    rom = rom.copy()
    rom[1:-1] = _away_from_zero(rom[1:-1], 10.0)
    xs = [dev(a).requires_grad_(True) for a in (q, ru, rv, rom)]

    def J(q_, ru_, rv_, rom_):
        y = adjoint.scalar_advection(q_, ru_, rv_, rom_, nl)
        return 0.5 * (y * y).sum()

    grads = torch.autograd.grad(J(*xs), xs)
    # the fused launch's q cotangent is the q-only adjoint's, bit for bit
    q_only = dev(q).requires_grad_(True)
    (g_q,) = torch.autograd.grad(J(q_only, *(dev(a) for a in (ru, rv, rom))), q_only)
    assert torch.equal(g_q, grads[0])
    rng = np.random.default_rng(9)
    ds = [rng.standard_normal(a.shape) for a in (q, ru, rv, rom)]
    ds[3][0] = 0.0
    ds[3][-1] = 0.0
    scale = [1.0, 5.0e4, 5.0e4, 1.0e3]  # perturb each input in proportion to its size
    h = 1.0e-4
    plus = [dev(a + h * s * d) for a, s, d in zip((q, ru, rv, rom), scale, ds)]
    minus = [dev(a - h * s * d) for a, s, d in zip((q, ru, rv, rom), scale, ds)]
    fd = (float(J(*plus)) - float(J(*minus))) / (2 * h)
    ad = sum(float((g * dev(s * d)).sum()) for g, s, d in zip(grads, scale, ds))
    assert abs(fd - ad) <= 1.0e-7 * abs(ad), (fd, ad)

