"""The y-slab decomposition of the step (``wrf_gpu_b200.sharding``) on the
CPU: the slab geometry and halo plan, and the decomposition driven in one
process with the oracle as each slab's step, against the oracle's
whole-domain step -- owned rows bit for bit, periodic and specified domains,
with the 6th-order and Smagorinsky filters (whose rolls wrap the domain
edges), the boundary cadence and the end-of-step boundary pass."""

from __future__ import annotations

import numpy as np
import pytest

from tests import sharding_util as SU
from wrf_gpu_b200 import cases, sharding

FIELDS = ("u", "v", "w", "theta", "p_total", "p_perturbation", "ph_total", "ph_perturbation", "mu_total",
          "mu_perturbation", "qv", "qc", "qr")


@pytest.mark.parametrize("ny,world,halo", [(90, 3, 19), (90, 2, 24), (100, 4, 24), (61, 3, 17), (40, 1, 30)])
def test_layout_covers_each_row_once_as_owned_and_places_the_halos(ny, world, halo):
    owned = np.zeros(ny, int)
    for r in range(world):
        L = sharding.slab_layout(ny, world, r, halo)
        rows = np.asarray(L.rows)
        assert L.n_local == (ny if world == 1 else L.own + 2 * halo)
        np.testing.assert_array_equal(rows[L.own_local:L.own_local + L.own], np.arange(L.own_lo, L.own_hi))
        owned[L.own_lo:L.own_hi] += 1
        if world == 1:
            continue
        np.testing.assert_array_equal(rows[L.below_local:L.below_local + halo],
                                      np.arange(L.own_lo - halo, L.own_lo) % ny)
        np.testing.assert_array_equal(rows[L.above_local:L.above_local + halo],
                                      np.arange(L.own_hi, L.own_hi + halo) % ny)
        # the domain's edges sit at the slab's edges whenever the slab holds them
        if 0 in rows:
            assert rows[0] == 0 and rows[-1] == ny - 1
        assert L.faces()[-1] == rows[-1] + 1
    np.testing.assert_array_equal(owned, 1)


def test_send_and_receive_blocks_match_between_neighbours():
    world, ny, H = 3, 90, 19
    case = cases.real_like_moist(12, ny, 6, hmax=100.0, specified=False)
    nl = SU.host_namelist(case)
    slabs = [sharding.SlabStepper(nl, sharding.slab_layout(ny, world, r, H), copier=SU.TorchRows(),
                                  step_fn=lambda c, n, l: c) for r in range(world)]
    carry = SU.host_carry(case)
    for s in slabs:
        s.load(carry)
    for s in slabs:
        (below, nb), (above, na) = s.recv_blocks()
        (_, n_down), (_, n_up) = slabs[s.layout.below].send_blocks()[0], slabs[s.layout.below].send_blocks()[1]
        assert nb == n_up  # the rank below sends its top rows up
        assert na == slabs[s.layout.above].send_blocks()[0][1]  # the rank above sends its bottom rows down
        # the block from below that ends at the domain's top row carries the north face of v
        v_rows = {b[2] for b in below if b[0] is s.carry.state.v}
        assert v_rows == ({H + 1} if s.layout.rank == 0 else {H})


def test_halo_rows_and_rejections():
    spec = SU.host_namelist(cases.real_like_moist(12, 40, 6, hmax=100.0, specified=True))
    per = SU.host_namelist(cases.real_like_moist(12, 40, 6, hmax=100.0, specified=False))
    assert sharding.halo_rows(per) == 10 + 6 + 3
    assert sharding.halo_rows(spec) == 10 + 6 + 3 + 1 + 4
    from dataclasses import replace
    with pytest.raises(NotImplementedError):
        sharding.halo_rows(replace(per, const_nu_m2_s=10.0))
    with pytest.raises(ValueError):
        sharding.slab_layout(40, 3, 0, 19)


def _case(specified, ny=90, **controls):
    c = cases.real_like_moist(16, ny, 8, hmax=300.0, ns=6, specified=specified, bdy_noise=specified)
    if specified:
        c = cases.with_full_leaves(c, rng=np.random.default_rng(5))
    c.controls.update(controls)
    return c


def _ring(case, world, nsteps, halo=None, boundary_pass=False):
    nl = SU.host_namelist(case)
    ring = sharding.SlabRing(nl, world, halo=halo, boundary_pass=boundary_pass, copier=SU.TorchRows(),
                             step_fn=SU.oracle_step_fn(case, boundary_pass))
    ring.load(SU.host_carry(case))
    for i in range(nsteps):
        ring.step((i + 1) * nl.dt_s)
    return ring.gather()


@pytest.mark.parametrize("specified,world,controls,boundary_pass", [
    (False, 3, {}, False),
    (False, 2, {"diff_6th_opt": 2, "diff_opt": 1, "km_opt": 4}, False),
    (True, 3, {"specified_bdy_cadence": True, "diff_6th_opt": 2, "diff_opt": 1, "km_opt": 4}, True),
    (True, 2, {}, True),
])
def test_slab_ring_matches_the_whole_domain_bit_for_bit(specified, world, controls, boundary_pass):
    case = _case(specified, **controls)
    got = _ring(case, world, 3, boundary_pass=boundary_pass)
    want = SU.oracle_run(case, 3, boundary_pass)
    for f in FIELDS:
        np.testing.assert_array_equal(getattr(got.state, f).numpy(), getattr(want.state, f), err_msg=f)
    np.testing.assert_array_equal(got.mudf.numpy(), want.mudf)


def test_a_halo_narrower_than_one_step_reach_breaks_the_match():
    case = _case(True, specified_bdy_cadence=True)
    got = _ring(case, 3, 2, halo=12)
    want = SU.oracle_run(case, 2)
    assert not np.array_equal(got.state.w.numpy(), want.state.w)
