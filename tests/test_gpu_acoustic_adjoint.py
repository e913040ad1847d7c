"""The standalone acoustic small step and its hand-written vector-Jacobian
product (``wrfgpu_acoustic_substep[_vjp]``, ``adjoint.AcousticOp``).

* forward parity: one CUDA substep against the oracle's ``acoustic_substep``
  on the work state and stage constants the oracle's RK stage builds (doubly
  periodic; and specified, with the relax-zone blend, the frozen ring and
  the drain limiter), per field at the per-step tolerance;
* adjoint: the dot-product identity <cot_out, J d> = <J^T cot_out, d>, with
  J d from central finite differences of the oracle's float64 substep (and of
  the CUDA substep), for all fields together and one input field at a time;
  the FD step is 1e-5 (1e-3 per field) of each field's spread, so the
  identity holds to ~1e-8.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import dycore as D
from tests import parity_util as P
from wrf_gpu_b200 import _capi, adjoint, cases, dycore

pytestmark = pytest.mark.gpu

# C work-state names -> oracle attribute names
WORK = dict(zip(_capi.ACOUSTIC_WORK_FIELDS, ("u", "v", "w", "ph", "theta_work", "t_2ave", "p", "pm1", "al", "ww",
                                              "mu", "muts", "muave", "mudf")))
CONSTS = {"u_tend": "u_tend", "v_tend": "v_tend", "t_tend": "theta_tend", "rw_tend": "rw_tend",
          "ph_tend": "ph_tend", "alt": "alt", "pb": "pb", "c2a": "c2a", "cqu": "cqu", "cqv": "cqv", "cqw": "cqw",
          "php": "php", "a": "a", "alpha": "alpha", "gamma": "gamma", "ww_1": "ww_1", "mut": "mut", "muu": "muu",
          "muv": "muv", "mu_tend": "mu_tend", "u_1": "u_1", "v_1": "v_1", "w_save": "w_save"}
TOL = 1.0e-12


def _case(kind):
    if kind == "moist_periodic":
        case = cases.real_like_moist(24, 20, 12, hmax=800.0, specified=False)
    elif kind == "moist_specified":
        case = cases.real_like_moist(24, 20, 12, hmax=800.0, specified=True, bdy_noise=True)
    else:  # rigid lid, Rayleigh damping, stretched levels over terrain, made periodic
        case = cases.mountain_wave(24, 20, 14)
        case.controls.update(run_boundary=False, bc_ideal=True, top_lid=True)
    return case


def _stage(case, rk):
    nl = P.oracle_namelist(case)
    out = P.oracle_steps(case, 1)  # a developed flow
    carry = SimpleNamespace(state=out.state, mudf=out.mudf)
    lead = nl.dt_s if nl.run_boundary else None
    a, dts, s, bdy = D.stage_acoustic_state(carry, nl, rk, lead)
    a.bdy = bdy
    return nl, a, dts, s


def _op(case, a, s, dts):
    dev = lambda x: torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device="cuda")
    consts = {k: dev(getattr(a, v)) for k, v in CONSTS.items()}
    consts["pt1"] = dev(a.ph_1 + a.phb)
    consts["theta"] = dev(s.theta)
    consts["phb0"] = dev(a.phb[0])
    if a.bdy is not None:
        consts["u_target"], consts["v_target"] = dev(a.bdy.u_target), dev(a.bdy.v_target)
    nlg = dycore.OperationalNamelist.from_case(case)
    return adjoint.AcousticOp(nlg, consts, dts)


def _oracle_step(nl, a, dts, x):
    b = D.copy_state(a)
    for cn, on in WORK.items():
        setattr(b, on, x[cn].copy())
    D.acoustic_substep(b, nl.metrics, nl, dts, a.bdy)
    return {cn: getattr(b, on) for cn, on in WORK.items()}


def _cuda_step(op, x):
    ts = [torch.as_tensor(x[n].copy(), device="cuda") for n in _capi.ACOUSTIC_WORK_FIELDS]
    op.forward_(ts)
    torch.cuda.synchronize()
    return {n: t.cpu().numpy() for n, t in zip(_capi.ACOUSTIC_WORK_FIELDS, ts)}


def _dot(a, b):
    return sum(float(np.sum(a[n] * b[n])) for n in a)


@pytest.mark.parametrize("kind,rk", [("moist_periodic", 3), ("moist_periodic", 1), ("lid_damped", 3),
                                     ("moist_specified", 3), ("moist_specified", 1)])
def test_substep_forward_matches_oracle(cuda_ready, kind, rk):
    case = _case(kind)
    nl, a, dts, s = _stage(case, rk)
    x = {cn: getattr(a, on).copy() for cn, on in WORK.items()}
    op = _op(case, a, s, dts)
    got = _cuda_step(op, x)
    want = _oracle_step(nl, a, dts, x)
    for n in _capi.ACOUSTIC_WORK_FIELDS:
        err = P.rel_err(got[n], want[n])
        assert err <= TOL, (n, err)


@pytest.mark.parametrize("kind", ["moist_periodic", "lid_damped", "moist_specified"])
def test_substep_vjp_dot_product_against_finite_differences(cuda_ready, kind):
    case = _case(kind)
    nl, a, dts, s = _stage(case, 3)
    x = {cn: getattr(a, on).copy() for cn, on in WORK.items()}
    op = _op(case, a, s, dts)
    rng = np.random.default_rng(20261203)
    y = _oracle_step(nl, a, dts, x)
    spread = lambda f: float(np.std(f)) + 1.0e-3 * (float(np.max(np.abs(f))) + 1.0)
    # directions on each field's own scale (the stage-start work u, v, w, ww are zero: use the output's)
    d = {n: rng.standard_normal(x[n].shape) * max(spread(x[n]), spread(y[n])) for n in x}
    cot = {n: rng.standard_normal(y[n].shape) / spread(y[n]) for n in y}
    ts = [torch.as_tensor(x[n], device="cuda") for n in _capi.ACOUSTIC_WORK_FIELDS]
    cs = [torch.as_tensor(cot[n], device="cuda") for n in _capi.ACOUSTIC_WORK_FIELDS]
    ci = op.vjp(ts, cs)
    # with the stored forward output instead of the recomputed one: the same cotangents
    outs = [t.clone() for t in ts]
    op.forward_(outs)
    ci_stored = op.vjp(ts, cs, outs)
    torch.cuda.synchronize()
    ci = {n: t.cpu().numpy() for n, t in zip(_capi.ACOUSTIC_WORK_FIELDS, ci)}
    # the cotangents are summed in a fixed order: bit for bit the same
    for n, t in zip(_capi.ACOUSTIC_WORK_FIELDS, ci_stored):
        assert np.array_equal(t.cpu().numpy(), ci[n]), n
    # muave enters no output of an updated column (a specified domain's frozen ring passes it through)
    inner = (slice(1, -1), slice(1, -1)) if a.bdy is not None else (slice(None), slice(None))
    assert np.all(ci["muave"][inner] == 0.0)
    h = 1.0e-5

    def jd(step, dd):
        xp = {n: x[n] + h * dd[n] for n in x}
        xm = {n: x[n] - h * dd[n] for n in x}
        fp, fm = step(xp), step(xm)
        return {n: (fp[n] - fm[n]) / (2.0 * h) for n in fp}

    oracle = lambda xx: _oracle_step(nl, a, dts, xx)
    cuda = lambda xx: _cuda_step(op, xx)
    for step in (oracle, cuda):
        lhs, rhs = _dot(cot, jd(step, d)), _dot(ci, d)
        assert abs(lhs - rhs) <= 1.0e-8 * (abs(lhs) + abs(rhs)), (lhs, rhs)
    # one input field at a time against the oracle's derivative, with a
    # longer FD step (the step is affine in every field but muts, whose
    # curvature is ~1e-9 at this step) over the FD's rounding floor of
    # ~eps |cot| |y| / h summed over the outputs
    h = 1.0e-3
    floor = 8.0 * np.finfo(np.float64).eps / (2.0 * h) * sum(float(np.sum(np.abs(cot[n] * y[n]))) for n in y)
    for n in _capi.ACOUSTIC_WORK_FIELDS:
        dn = {m: (d[m] if m == n else np.zeros_like(d[m])) for m in d}
        lhs, rhs = _dot(cot, jd(oracle, dn)), float(np.sum(ci[n] * d[n]))
        assert abs(lhs - rhs) <= 1.0e-8 * (abs(lhs) + abs(rhs)) + floor, (n, lhs, rhs, floor)


def test_autograd_function_chains_two_substeps(cuda_ready):
    case = _case("moist_periodic")
    nl, a, dts, s = _stage(case, 3)
    op = _op(case, a, s, dts)
    x = {cn: torch.as_tensor(getattr(a, on).copy(), device="cuda").requires_grad_(True) for cn, on in WORK.items()}
    y = adjoint.acoustic_substep(adjoint.acoustic_substep(x, op), op)
    loss = (y["w"] ** 2).sum() + (y["theta_w"] ** 2).sum() * 1.0e-4
    loss.backward()
    rng = np.random.default_rng(5)
    d = {n: torch.as_tensor(rng.standard_normal(tuple(t.shape)) * (float(t.detach().std()) + 1e-3), device="cuda")
         for n, t in x.items()}
    h = 1.0e-5

    def f(sign):
        with torch.no_grad():
            z = {n: x[n].detach() + sign * h * d[n] for n in x}
            z = adjoint.acoustic_substep(adjoint.acoustic_substep(z, op), op)
            return float((z["w"] ** 2).sum() + (z["theta_w"] ** 2).sum() * 1.0e-4)

    fd = (f(1.0) - f(-1.0)) / (2.0 * h)
    ad = sum(float((x[n].grad * d[n]).sum()) for n in x)
    assert abs(fd - ad) <= 1.0e-6 * abs(ad), (fd, ad)


def _tiled_op(n, nz=50):
    """Stage constants and work state at n x n x nz tiled from an oracle stage
    of the periodic real-like moist case (timing is data independent)."""
    small = cases.real_like_moist(24, 20, nz, hmax=800.0, specified=False)
    nl = P.oracle_namelist(small)
    carry = SimpleNamespace(state=D.copy_state(small.state), mudf=small.mudf.copy())
    a, dts, s, _ = D.stage_acoustic_state(carry, nl, 3)

    def fit(arr, ly, lx):
        arr = np.asarray(arr)
        reps = [1] * (arr.ndim - 2) + [-(-ly // arr.shape[-2]), -(-lx // arr.shape[-1])]
        return np.ascontiguousarray(np.tile(arr, reps)[..., :ly, :lx])

    xshape = {"u": (n, n + 1), "v": (n + 1, n), "cqu": (n, n + 1), "cqv": (n + 1, n), "u_tend": (n, n + 1),
              "v_tend": (n + 1, n), "u_1": (n, n + 1), "v_1": (n + 1, n), "muu": (n, n + 1), "muv": (n + 1, n)}
    dev = lambda arr: torch.as_tensor(arr, dtype=torch.float64, device="cuda")
    x = [dev(fit(getattr(a, WORK[k]), *xshape.get(k, (n, n)))) for k in _capi.ACOUSTIC_WORK_FIELDS]
    consts = {k: dev(fit(getattr(a, v), *xshape.get(k, (n, n)))) for k, v in CONSTS.items()}
    consts["pt1"] = dev(fit(a.ph_1 + a.phb, n, n))
    consts["theta"] = dev(fit(s.theta, n, n))
    consts["phb0"] = dev(fit(a.phb[0], n, n))
    big = cases.real_like_moist(n, n, nz, hmax=800.0, specified=False)
    return adjoint.AcousticOp(dycore.OperationalNamelist.from_case(big), consts, dts), x


def test_vjp_cost_relative_to_forward(cuda_ready):
    op, x = _tiled_op(433)
    co = [torch.randn_like(t) for t in x]

    def timed(fn, reps=10):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    xs = [t.clone() for t in x]
    t_fwd = timed(lambda: op.forward_(xs))
    t_vjp = timed(lambda: op.vjp(x, co))
    xo = [t.clone() for t in x]
    op.forward_(xo)
    t_st = timed(lambda: op.vjp(x, co, xo))
    print(f"acoustic substep at 433x433x50: forward {t_fwd:.3f} ms, VJP {t_vjp:.3f} ms ({t_vjp / t_fwd:.2f}x) "
          f"recomputing the forward output, {t_st:.3f} ms ({t_st / t_fwd:.2f}x) from the stored one")
    assert t_st <= 3.0 * t_fwd
    assert t_vjp <= 3.0 * t_fwd  # the checkpointing mode: forward recomputed inside the VJP


def test_checkpointed_loop_matches_chained_substeps(cuda_ready):
    case = _case("lid_damped")
    nl, a, dts, s = _stage(case, 3)
    op = _op(case, a, s, dts)
    base = {cn: torch.as_tensor(getattr(a, on).copy(), device="cuda") for cn, on in WORK.items()}

    def loss(y):
        return (y["w"] ** 2).sum() + 1.0e-4 * (y["theta_w"] ** 2).sum() + 1.0e-2 * (y["p"] ** 2).sum()

    x1 = {n: t.clone().requires_grad_(True) for n, t in base.items()}
    y1 = x1
    for _ in range(3):
        y1 = adjoint.acoustic_substep(y1, op)
    loss(y1).backward()
    x2 = {n: t.clone().requires_grad_(True) for n, t in base.items()}
    y2 = adjoint.acoustic_loop(x2, op, 3)
    for n in y1:
        assert torch.equal(y1[n], y2[n]), n
    loss(y2).backward()
    for n in x1:
        g1, g2 = x1[n].grad, x2[n].grad
        scale = float(g1.abs().max()) or 1.0
        assert float((g1 - g2).abs().max()) <= 1.0e-12 * scale, n


# C tendency-cotangent names -> oracle attribute names
TENDS = {"u_tend": "u_tend", "v_tend": "v_tend", "t_tend": "theta_tend", "rw_tend": "rw_tend", "ph_tend": "ph_tend",
         "mu_tend": "mu_tend"}


@pytest.mark.parametrize("kind", ["moist_periodic", "lid_damped", "moist_specified"])
def test_substep_vjp_tendency_cotangents(cuda_ready, kind):
    """The cotangents of the stage tendencies against central differences of
    the oracle's substep in each tendency (all together and one at a time)."""
    case = _case(kind)
    nl, a, dts, s = _stage(case, 3)
    x = {cn: getattr(a, on).copy() for cn, on in WORK.items()}
    op = _op(case, a, s, dts)
    rng = np.random.default_rng(99)
    y = _oracle_step(nl, a, dts, x)
    spread = lambda f: float(np.std(f)) + 1.0e-3 * (float(np.max(np.abs(f))) + 1.0)
    cot = {n: rng.standard_normal(y[n].shape) / spread(y[n]) for n in y}
    ts = [torch.as_tensor(x[n], device="cuda") for n in _capi.ACOUSTIC_WORK_FIELDS]
    cs = [torch.as_tensor(cot[n], device="cuda") for n in _capi.ACOUSTIC_WORK_FIELDS]
    _, tc = op.vjp(ts, cs, tendencies=True)
    torch.cuda.synchronize()
    tc = {n: t.cpu().numpy() for n, t in tc.items()}
    d = {n: rng.standard_normal(np.shape(getattr(a, on))) * spread(np.asarray(getattr(a, on)) + 1.0)
         for n, on in TENDS.items()}
    h = 1.0e-3

    def jd(dd):
        def step(sign):
            b = D.copy_state(a)
            for n, on in TENDS.items():
                setattr(b, on, np.asarray(getattr(a, on)) + sign * h * dd[n])
            return _oracle_step(nl, b, dts, x)
        fp, fm = step(1.0), step(-1.0)
        return {n: (fp[n] - fm[n]) / (2.0 * h) for n in fp}

    floor = 8.0 * np.finfo(np.float64).eps / (2.0 * h) * sum(float(np.sum(np.abs(cot[n] * y[n]))) for n in y)
    lhs, rhs = _dot(cot, jd(d)), sum(float(np.sum(tc[n] * d[n])) for n in d)
    assert abs(lhs - rhs) <= 1.0e-8 * (abs(lhs) + abs(rhs)) + floor, (lhs, rhs)
    for n in TENDS:
        dn = {m: (d[m] if m == n else np.zeros_like(d[m])) for m in d}
        lhs, rhs = _dot(cot, jd(dn)), float(np.sum(tc[n] * d[n]))
        assert abs(lhs - rhs) <= 1.0e-8 * (abs(lhs) + abs(rhs)) + floor, (n, lhs, rhs, floor)


def test_vjp_is_bitwise_reproducible(cuda_ready):
    """The advance_uv transpose gathers every cell's face shares in a fixed
    order (no atomic accumulation): repeated VJPs are identical bit for bit."""
    case = _case("moist_specified")
    nl, a, dts, s = _stage(case, 3)
    x = {cn: getattr(a, on).copy() for cn, on in WORK.items()}
    op = _op(case, a, s, dts)
    rng = np.random.default_rng(7)
    ts = [torch.as_tensor(x[n], device="cuda") for n in _capi.ACOUSTIC_WORK_FIELDS]
    cs = [torch.as_tensor(rng.standard_normal(x[n].shape), device="cuda") for n in _capi.ACOUSTIC_WORK_FIELDS]
    runs = [[t.cpu().numpy() for t in op.vjp(ts, cs)] for _ in range(3)]
    for r in runs[1:]:
        for n, a0, a1 in zip(_capi.ACOUSTIC_WORK_FIELDS, runs[0], r):
            assert np.array_equal(a0, a1), n
