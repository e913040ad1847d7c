"""The hand-written adjoint of the flux-form scalar advection operator.

* forward: the CUDA operator against the oracle's advect_scalar_flux
  (flux_advection.py:482-568) on random fields and velocities, 1e-12;
* adjoint: the dot-product identity <L q, lam> = <q, L^T lam> to 1e-12
  relative, and central finite differences of J(q) = 0.5 |L q|^2 along random
  directions against <grad J, d> from torch autograd (1e-8: the operator is
  linear, so the differences are exact up to rounding);
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
