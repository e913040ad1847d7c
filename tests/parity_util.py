"""Shared helpers for the parity tests: run the oracle and the CUDA step on the
same seeded case and compare every prognostic and carry field."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import dycore as D

STATE_KEYS = ("u", "v", "w", "theta", "p_total", "p_perturbation", "ph_total", "ph_perturbation",
              "mu_total", "mu_perturbation", "qv", "qc", "qr", "qi", "qs", "qg")
CARRY_KEYS = ("t_2ave", "ww", "mudf", "muave", "muts", "ph_tend", "u_save", "v_save", "w_save", "t_save",
              "ph_save", "mu_save", "ww_save")


def oracle_namelist(case):
    return D.Namelist(metrics=case.metrics, **case.controls)


def oracle_steps(case, nsteps, lead0=0.0, physics=None):
    nl = oracle_namelist(case)
    carry = SimpleNamespace(state=D.copy_state(case.state), mudf=case.mudf.copy())
    for i in range(nsteps):
        carry = D.rk_scan_step(carry, nl, lead_seconds=lead0 + i * nl.dt_s, physics=physics)
    return carry


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    diff = float(np.max(np.abs(a - b))) if b.size else 0.0
    if scale == 0.0:
        return diff
    return diff / scale


def compare(gpu_carry, ora_carry, keys_state=STATE_KEYS, keys_carry=CARRY_KEYS):
    out = {}
    gs = gpu_carry.state
    for k in keys_state:
        g = getattr(gs, k, None)
        o = getattr(ora_carry.state, k, None)
        if g is None or o is None:
            continue
        out[k] = rel_err(g.cpu().numpy(), o)
    for k in keys_carry:
        g = getattr(gpu_carry, k, None)
        o = getattr(ora_carry, k, None)
        if g is None or o is None:
            continue
        out[k] = rel_err(g.cpu().numpy(), o)
    return out


def attach_lbc_leaves(s, rng, moist=("qv", "qc", "qr")):
    """Drifting random strips (2 times) for the leaves a real-like case does
    not carry (p, pb, mub, phb) and for ``moist`` (a few negatives, for the
    clip); shapes (2, 4, 5, levels, side_len)."""
    nz = s.theta.shape[0]
    side = s.u_bdy.shape[-1]
    leaf = lambda z, mean, sc: mean + sc * rng.standard_normal((2, 4, 5, z, side))
    s.p_bdy, s.pb_bdy = leaf(nz, 0.0, 40.0), leaf(nz, 5.0e4, 100.0)
    s.mub_bdy, s.phb_bdy = leaf(1, 9.0e4, 50.0), leaf(nz + 1, 2.0e4, 20.0)
    for q in moist:
        setattr(s, q + "_bdy", np.abs(leaf(nz, 1.0e-3, 1.0e-3)) - 2.0e-4)
    return s


def compare_oracles(a, b, keys_state=STATE_KEYS, keys_carry=CARRY_KEYS):
    """``compare`` for two oracle carries (host arrays on both sides)."""
    out = {}
    for k in keys_state:
        x, y = getattr(a.state, k, None), getattr(b.state, k, None)
        if x is not None and y is not None:
            out[k] = rel_err(x, y)
    for k in keys_carry:
        x, y = getattr(a, k, None), getattr(b, k, None)
        if x is not None and y is not None:
            out[k] = rel_err(x, y)
    return out
