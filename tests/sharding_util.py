"""Test doubles for the y-slab decomposition on host tensors: a row mover
by tensor slicing and a slab step by the oracle, so that the decomposition,
the halo plan and the exchange run on the CPU (in one process, or as gloo
ranks) against the oracle's whole-domain step."""

from __future__ import annotations

from dataclasses import fields
from types import SimpleNamespace

import numpy as np
import torch

from oracle import dycore as D
from wrf_gpu_b200 import dycore

CARRY_OUT = ("t_2ave", "ww", "mudf", "muave", "muts", "ph_tend", "u_save", "v_save", "w_save", "t_save", "ph_save",
             "mu_save", "ww_save")


def _as3(t):
    return t if t.dim() == 3 else t.unsqueeze(0)


class TorchRows:
    """Row copies, packs and unpacks by slicing (host tensors)."""

    def copy(self, src, src_row0, dst, dst_row0, nrows, stream=None):
        _as3(dst)[:, dst_row0:dst_row0 + nrows] = _as3(src)[:, src_row0:src_row0 + nrows]

    def pack(self, blocks, buffer, stream=None):
        for t, row0, nrows, off in blocks:
            b = _as3(t)[:, row0:row0 + nrows]
            buffer[off:off + b.numel()] = b.reshape(-1)

    def unpack(self, blocks, buffer, stream=None):
        for t, row0, nrows, off in blocks:
            t3 = _as3(t)
            n = t3.shape[0] * nrows * t3.shape[2]
            t3[:, row0:row0 + nrows] = buffer[off:off + n].reshape(t3.shape[0], nrows, t3.shape[2])


def oracle_step_fn(case, boundary_pass=False):
    """A slab step by the oracle: the slab's namelist (its metrics rows) with
    the case's controls; with ``boundary_pass`` the end-of-step lateral
    boundary pass as the forecast step runs it (guards off)."""

    def step(carry, nl, lead):
        m = nl.metrics
        om = SimpleNamespace(**vars(case.metrics))
        for n in dycore.METRIC_ARRAYS:
            setattr(om, n, getattr(m, n).numpy())
        onl = D.Namelist(metrics=om, **case.controls)
        s = SimpleNamespace(**{k: v.numpy() for k, v in vars(carry.state).items() if v is not None})
        origin = s
        nxt = D.rk_scan_step(SimpleNamespace(state=D.copy_state(s), mudf=carry.mudf.numpy()), onl,
                             lead_seconds=lead)
        state = nxt.state
        if boundary_pass and onl.run_boundary:
            spec_only = onl.specified_bdy_cadence and not onl.bc_ideal and onl.force_geopotential
            state, _ = D.step_epilogue(nxt.state, origin, lead, onl.dt_s, onl, run_boundary=True,
                                       dry_spec_only=spec_only, disable_guards=True)
        st = dycore.State(**{f.name: (torch.from_numpy(np.ascontiguousarray(getattr(state, f.name)))
                                      if getattr(state, f.name, None) is not None else None)
                             for f in fields(dycore.State)})
        return dycore.OperationalCarry(state=st, **{n: torch.from_numpy(np.ascontiguousarray(getattr(nxt, n)))
                                                    for n in CARRY_OUT})

    return step


def host_carry(case):
    st = dycore.State.from_host(case.state, device="cpu")
    return dycore.initial_operational_carry(st).replace(mudf=torch.from_numpy(case.mudf.copy()))


def host_namelist(case):
    return dycore.OperationalNamelist.from_case(case, device="cpu")


def oracle_run(case, nsteps, boundary_pass=False):
    nl = D.Namelist(metrics=case.metrics, **case.controls)
    carry = SimpleNamespace(state=D.copy_state(case.state), mudf=case.mudf.copy())
    for i in range(nsteps):
        lead = (i + 1) * nl.dt_s
        origin = carry.state
        nxt = D.rk_scan_step(carry, nl, lead_seconds=lead)
        state = nxt.state
        if boundary_pass and nl.run_boundary:
            spec_only = nl.specified_bdy_cadence and not nl.bc_ideal and nl.force_geopotential
            state, _ = D.step_epilogue(nxt.state, origin, lead, nl.dt_s, nl, run_boundary=True,
                                       dry_spec_only=spec_only, disable_guards=True)
        carry = SimpleNamespace(state=state, mudf=nxt.mudf)
    return carry
