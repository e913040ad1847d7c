"""The distributed form of the y-slab decomposition (``DistributedSlab``)
as two gloo ranks on the CPU: each rank steps its slab with the oracle,
swaps halo blocks with its neighbour by point-to-point messages (both
neighbours are the same peer with two ranks, so the message order matters)
and all-gathers the owned rows; both ranks must hold the oracle's
whole-domain result bit for bit."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

FIELDS = ("u", "v", "w", "theta", "p_perturbation", "ph_perturbation", "mu_perturbation", "qv", "mudf")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(specified):
    from wrf_gpu_b200 import cases
    c = cases.real_like_moist(16, 80, 8, hmax=300.0, ns=6, specified=specified, bdy_noise=specified)
    if specified:
        c = cases.with_full_leaves(c, rng=np.random.default_rng(5))
        c.controls.update(specified_bdy_cadence=True, diff_6th_opt=2)
    return c


def _rank(rank, world, port, specified, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from tests import sharding_util as SU
        from wrf_gpu_b200 import sharding
        case = _case(specified)
        nl = SU.host_namelist(case)
        ds = sharding.DistributedSlab(nl, copier=SU.TorchRows(), step_fn=SU.oracle_step_fn(case, specified),
                                      boundary_pass=specified)
        ds.load(SU.host_carry(case))
        for i in range(3):
            ds.step((i + 1) * nl.dt_s)
        g = ds.gather()
        want = SU.oracle_run(case, 3, specified)
        bad = []
        for f in FIELDS:
            a = (g.mudf if f == "mudf" else getattr(g.state, f)).numpy()
            b = want.mudf if f == "mudf" else getattr(want.state, f)
            if not np.array_equal(a, b):
                bad.append((f, float(np.max(np.abs(a - b)))))
        q.put((rank, ds.slab.layout.halo, bad))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("specified", [False, True])
def test_two_gloo_ranks_step_their_slabs_to_the_whole_domain_result(specified):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, specified, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, halo, bad in got:
        assert halo == (24 if specified else 19)
        assert not bad, (rank, bad)
