"""Device checks of the numerical helpers the kernels rely on.

``div_rcp(a, b, rb)`` replaces ``a / b`` for divisors with a precomputed
correctly rounded reciprocal (the flux stencils' 1/60 and 1/12, the upwind
fluxes' dx, dy and dz).  It must reproduce CUDA's IEEE division bit for bit,
so the kernels keep the reference's rounding.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from wrf_gpu_b200 import build

pytestmark = pytest.mark.gpu


def _selftest_lib():
    build.build()
    lib = ctypes.CDLL(str(build.SELFTEST_LIB))
    f = lib.wrfgpu_selftest_div_rcp
    f.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_long, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _random_doubles(rng, n, emin, emax):
    mant = rng.integers(0, 1 << 52, size=n, dtype=np.uint64)
    exp = rng.integers(emin + 1023, emax + 1024, size=n, dtype=np.uint64)
    sign = rng.integers(0, 2, size=n, dtype=np.uint64)
    return ((sign << np.uint64(63)) | (exp << np.uint64(52)) | mant).view(np.float64)


def test_div_rcp_matches_cuda_division_bitwise(cuda_ready):
    f = _selftest_lib()
    rng = np.random.default_rng(7)
    n_per = 1 << 20
    divisors = [60.0, 12.0, 9.81, 6.0, 2.0 / 3.0, 1000.0, 1.0 / (1.0 / 3000.0), 1.0 / (1.0 / 333.3)]
    divisors += list(np.abs(_random_doubles(rng, 24, -30, 30)))
    for b in divisors:
        a = np.concatenate([_random_doubles(rng, n_per - 4, -600, 600), [0.0, 1.0, -1.0, 1.0e-20]])
        da = torch.as_tensor(a, device="cuda")
        db = torch.full_like(da, b)
        drb = torch.full_like(da, 1.0 / b)
        q1, q2 = torch.empty_like(da), torch.empty_like(da)
        rc = f(da.data_ptr(), db.data_ptr(), drb.data_ptr(), q1.data_ptr(), q2.data_ptr(), da.numel(),
               torch.cuda.current_stream().cuda_stream)
        assert rc == 0
        torch.cuda.synchronize()
        x, y = q1.cpu().numpy(), q2.cpu().numpy()
        same = (x.view(np.uint64) == y.view(np.uint64)) | ((x == 0.0) & (y == 0.0))
        assert same.all(), f"b={b!r}: {int((~same).sum())} mismatches, e.g. a={a[~same][:3]}"
