"""Host-side pieces of the advection adjoints that run without a GPU.

``adjoint.advect_w`` interpolates the transport velocities ru, rv from the
mass levels to w's levels before handing them to the flux operator
(flux_advection.py:1332-1352, the oracle's ``_mass_to_full``); that
interpolation is plain torch arithmetic, so it is checked here on the CPU
against the oracle, bit for bit, and its autograd transpose against the
adjoint identity.  The momentum operators' face averages (``advect_u`` /
``advect_v``) are torch rolls of the same kind and are covered by the GPU
parity tests.
"""

from __future__ import annotations

import numpy as np
import torch

from oracle import dycore as D
from wrf_gpu_b200 import adjoint, cases


def test_mass_to_full_matches_the_oracle_bit_for_bit():
    nz, ny, nx = 12, 7, 9
    m = cases.warm_bubble_3d(nx, ny, nz).metrics
    rng = np.random.default_rng(3)
    f = 1.0e4 * rng.standard_normal((nz, ny, nx))
    ora = D._mass_to_full(f, m.fnm, m.fnp)
    got = adjoint._mass_to_full(torch.as_tensor(f), torch.as_tensor(np.asarray(m.fnm)[:nz]),
                                torch.as_tensor(np.asarray(m.fnp)[:nz])).numpy()
    assert got.shape == (nz + 1, ny, nx)
    assert np.array_equal(got, ora)


def test_mass_to_full_transpose():
    """<P f, g> = <f, P^T g> for the autograd transpose of the interpolation."""
    nz, ny, nx = 10, 5, 6
    m = cases.warm_bubble_3d(nx, ny, nz).metrics
    rng = np.random.default_rng(4)
    fnm = torch.as_tensor(np.asarray(m.fnm)[:nz])
    fnp = torch.as_tensor(np.asarray(m.fnp)[:nz])
    f = torch.as_tensor(rng.standard_normal((nz, ny, nx)), dtype=torch.float64).requires_grad_(True)
    g = torch.as_tensor(rng.standard_normal((nz + 1, ny, nx)), dtype=torch.float64)
    y = adjoint._mass_to_full(f, fnm, fnp)
    (ft,) = torch.autograd.grad(y, f, grad_outputs=g)
    lhs = float((y.detach() * g).sum())
    rhs = float((f.detach() * ft).sum())
    assert abs(lhs - rhs) <= 1.0e-13 * max(abs(lhs), 1.0)
