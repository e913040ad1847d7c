"""The one-thread-per-column acoustic column kernel (``k_column_stream``,
selected by ``column_width = 1``) against the level-parallel one
(``k_column_tiled``, widths 16 / 32): the whole RK3 step must come out bit
for bit identical, on every branch the column kernel has -- periodic and
specified columns, the boundary cadence's and the nested child's ring-0 pins,
w damping, Rayleigh damping, the rigid lid, grids off every 32-column and
4-row multiple and a one-column slab."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from tests import parity_util as P
from wrf_gpu_b200 import cases, dycore

pytestmark = pytest.mark.gpu


def _step(case, width, lead=0.0):
    nl = dycore.OperationalNamelist.from_case(case)
    stp = dycore.Stepper(nl)
    stp.params.column_width = width
    a = dycore.carry_from_case(case)
    b = stp.alloc_carry(a)
    stp.step_into(a, b, lead_seconds=lead)
    torch.cuda.synchronize()
    return b


def _variants():
    out = []
    out.append(("periodic", cases.real_like_moist(37, 21, 14, hmax=800.0, specified=False)))
    out.append(("specified", cases.real_like_moist(45, 19, 14, hmax=800.0, specified=True)))
    c = cases.real_like_moist(40, 24, 12, hmax=800.0, specified=True, bdy_noise=True)
    c.controls.update(specified_bdy_cadence=True)
    out.append(("cadence", c))
    c = cases.real_like_moist(40, 24, 12, hmax=800.0, specified=True, bdy_noise=True)
    c.controls.update(force_geopotential=False, nested_ph_relax=True, nested_ph_spec=True)
    out.append(("nested", c))
    c = cases.real_like_moist(33, 17, 12, hmax=600.0, specified=False)
    c.controls.update(w_damping=1, damp_opt=3, dampcoef=0.2, zdamp=5000.0)
    out.append(("damping", c))
    c = cases.real_like_moist(33, 17, 12, hmax=600.0, specified=False)
    c.controls.update(top_lid=True)
    out.append(("top_lid", c))
    out.append(("mountain_wave", cases.mountain_wave(28, 24, 16)))
    out.append(("slab", cases.real_like_moist(1, 6, 5, hmax=300.0, specified=False)))
    out.append(("warm_bubble", cases.warm_bubble_3d(20, 16, 12)))
    return out


@pytest.mark.parametrize("name,case", _variants(), ids=[v[0] for v in _variants()])
def test_stream_column_kernel_is_bit_identical(cuda_ready, name, case):
    ref = _step(case, 32)
    for width in (1, 16):
        got = _step(case, width)
        for f in P.STATE_KEYS:
            a, b = getattr(ref.state, f), getattr(got.state, f)
            if a is None:
                continue
            assert torch.equal(a, b), (name, width, f, float((a - b).abs().max()))
        for f in P.CARRY_KEYS:
            assert torch.equal(getattr(ref, f), getattr(got, f)), (name, width, f)
