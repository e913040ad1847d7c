"""The y-slab decomposition on the device: the row-copy kernels against
tensor slicing, and every slab of a 2-, 3- and 4-way decomposition stepped
by the CUDA step in one process (``SlabRing``: the halo blocks packed by
``wrfgpu_rows_pack`` and unpacked into the neighbours by
``wrfgpu_rows_unpack``) against the whole-domain CUDA step, owned rows bit
for bit over three steps."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from wrf_gpu_b200 import _capi, cases, dycore, sharding

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "theta", "p_total", "p_perturbation", "ph_total", "ph_perturbation", "mu_total",
          "mu_perturbation", "qv", "qc", "qr")


def test_pack_unpack_and_copy_rows_match_slicing(cuda_ready):
    g = torch.Generator(device="cuda").manual_seed(3)
    a = torch.randn(7, 33, 21, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(33, 20, dtype=torch.float64, device="cuda", generator=g)
    rows = sharding.CudaRows()
    blocks = [(a, 5, 9, 0), (b, 30, 3, 7 * 9 * 21)]
    n = 7 * 9 * 21 + 3 * 20
    buf = torch.full((n + 5,), float("nan"), dtype=torch.float64, device="cuda")
    rows.pack(blocks, buf)
    torch.cuda.synchronize()
    assert torch.equal(buf[:7 * 9 * 21], a[:, 5:14].reshape(-1))
    assert torch.equal(buf[7 * 9 * 21:n], b[30:33].reshape(-1))
    a2, b2 = torch.zeros_like(a), torch.zeros_like(b)
    rows.unpack([(a2, 5, 9, 0), (b2, 30, 3, 7 * 9 * 21)], buf)
    c = torch.zeros(7, 12, 21, dtype=torch.float64, device="cuda")
    rows.copy(a, 20, c, 2, 10)
    torch.cuda.synchronize()
    assert torch.equal(a2[:, 5:14], a[:, 5:14]) and not a2[:, :5].any() and not a2[:, 14:].any()
    assert torch.equal(b2[30:], b[30:]) and not b2[:30].any()
    assert torch.equal(c[:, 2:12], a[:, 20:30]) and not c[:, :2].any()
    with pytest.raises(_capi.WrfGpuError):
        rows.pack([(a, 30, 9, 0)], buf)  # rows beyond the array
    with pytest.raises(_capi.WrfGpuError):
        rows.pack([(a, 0, 9, 10)], torch.empty(100, dtype=torch.float64, device="cuda"))  # beyond the buffer
    with pytest.raises(_capi.WrfGpuError):
        rows.copy(a, 30, c, 0, 5)


def _case(specified, **controls):
    c = cases.real_like_moist(48, 120, 20, hmax=500.0, ns=6, specified=specified, bdy_noise=specified)
    if specified:
        c = cases.with_full_leaves(c, rng=np.random.default_rng(9))
    c.controls.update(controls)
    return c


def _whole_domain(case, nsteps, boundary_pass):
    nl = dycore.OperationalNamelist.from_case(case)
    carry = dycore.carry_from_case(case)
    for i in range(nsteps):
        lead = (i + 1) * nl.dt_s
        nxt = dycore.rk_scan_step(carry, nl, lead_seconds=lead)
        if boundary_pass and nl.run_boundary:
            from dataclasses import replace
            st, _ = dycore.step_epilogue(nxt.state, carry.state, lead, replace(nl, disable_guards=True))
            nxt = nxt.replace(state=st)
        carry = nxt
    return carry


@pytest.mark.parametrize("specified,world,controls", [
    (False, 2, {}),
    (False, 4, {"diff_6th_opt": 2, "diff_opt": 1, "km_opt": 4}),
    (True, 3, {"specified_bdy_cadence": True, "diff_6th_opt": 2, "diff_opt": 1, "km_opt": 4}),
    (True, 4, {}),
])
def test_slab_ring_on_the_device_matches_the_whole_domain_step(cuda_ready, specified, world, controls):
    case = _case(specified, **controls)
    nl = dycore.OperationalNamelist.from_case(case)
    ring = sharding.SlabRing(nl, world, boundary_pass=specified)
    ring.load(dycore.carry_from_case(case))
    for i in range(3):
        ring.step((i + 1) * nl.dt_s)
    got = ring.gather()
    want = _whole_domain(case, 3, specified)
    torch.cuda.synchronize()
    for f in FIELDS:
        a, b = getattr(got.state, f), getattr(want.state, f)
        assert torch.equal(a, b), (f, float((a - b).abs().max()))
    assert torch.equal(got.mudf, want.mudf)
