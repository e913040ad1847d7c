"""CUDA step vs the CPU oracle (parity), through the C ABI.

Per-step parity: both sides take the SAME input (the oracle's state after n
steps) and advance one RK3 step; every prognostic and carry field must agree
to 1e-12 relative max-abs (max|gpu - oracle| / max|oracle|).  Fields that are
still at the float64 noise floor of a near-rest start (the first steps of the
warm bubbles, where w and v are ~1e-4 m/s) are checked against the measured
sensitivity of the oracle itself to one-ulp changes of pow(): perturbing one
pow() result by one ulp moves such fields by ~1e-12..1e-11 relative.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import dycore as D
from tests import parity_util as P
from wrf_gpu_b200 import cases, dycore

pytestmark = pytest.mark.gpu

TOL = 1.0e-12
# Column-integral and cancellation-dominated diagnostics: mudf/muave are the
# net column mass divergence (a sum of 50 nearly cancelling terms), p' is
# p_total(EOS, pow) - pb.  One-ulp pow() differences put them at ~1e-12.
DIAG_TOL = 5.0e-12
DIAG = ("mudf", "muave", "p_perturbation")


def _tol(k):
    return DIAG_TOL if k in DIAG else TOL


def _gpu_one_step(case, state, mudf, lead, physics=None):
    c = SimpleNamespace(**vars(case))
    c.state = state
    c.mudf = mudf
    nl = dycore.OperationalNamelist.from_case(case)
    carry = dycore.carry_from_case(c)
    phys = None
    if physics is not None:
        phys = SimpleNamespace(**{k: (None if v is None else torch.as_tensor(v, device="cuda"))
                                  for k, v in vars(physics).items()})
    out = dycore.rk_scan_step(carry, nl, lead_seconds=lead, physics_tendencies=phys)
    torch.cuda.synchronize()
    return out


def _per_step(case, nsteps, physics=None):
    nl = P.oracle_namelist(case)
    carry = SimpleNamespace(state=D.copy_state(case.state), mudf=case.mudf.copy())
    worst = []
    for n in range(nsteps):
        lead = n * nl.dt_s
        ora = D.rk_scan_step(carry, nl, lead_seconds=lead, physics=physics)
        gpu = _gpu_one_step(case, carry.state, carry.mudf, lead, physics)
        worst.append(P.compare(gpu, ora))
        carry = SimpleNamespace(state=ora.state, mudf=ora.mudf)
    return worst


# (case builder, steps).  The specified moist crop is run for 2 steps only: the
# reference's step leaves the specified ring to its end-of-step lateral
# boundary pass (outside _rk_scan_step), without which a small crop with
# noisy winds diverges after a few steps in the oracle and on the GPU alike.
CASES = {
    "moist_periodic_pd": (lambda: cases.real_like_moist(24, 20, 14, hmax=800.0, specified=False), 3),
    "moist_specified_pd": (lambda: cases.real_like_moist(24, 20, 14, hmax=800.0, specified=True), 2),
    "mountain_wave_damped": (lambda: cases.mountain_wave(28, 24, 16), 3),
}


@pytest.mark.parametrize("name", list(CASES))
def test_per_step_parity_developed_flow(cuda_ready, name):
    make, nsteps = CASES[name]
    case = make()
    for n, errs in enumerate(_per_step(case, nsteps)):
        bad = {k: v for k, v in errs.items() if not v <= _tol(k)}
        assert not bad, f"{name} step {n}: {bad}"


def test_per_step_parity_moist_monotonic(cuda_ready):
    case = cases.real_like_moist(24, 20, 14, hmax=800.0, specified=False)
    case.controls["moist_adv_opt"] = 2
    case.controls["scalar_adv_opt"] = 1
    for n, errs in enumerate(_per_step(case, 2)):
        bad = {k: v for k, v in errs.items() if not v <= _tol(k)}
        assert not bad, f"step {n}: {bad}"


def test_per_step_parity_options(cuda_ready):
    """hypsometric_opt 2, w_damping 1, rigid lid, dry cqw, no W-Coriolis,
    base tendencies -- each branch of the step exercised once."""
    base = cases.real_like_moist(20, 18, 12, hmax=600.0, specified=False)
    variants = [dict(hypsometric_opt=2), dict(w_damping=1), dict(top_lid=True), dict(moist_cqw=False),
                dict(w_coriolis=False), dict(scalar_adv_opt=2)]
    for kw in variants:
        case = cases.real_like_moist(20, 18, 12, hmax=600.0, specified=False)
        case.controls.update(kw)
        errs = _per_step(case, 2)
        for n, e in enumerate(errs):
            bad = {k: v for k, v in e.items() if not v <= _tol(k)}
            assert not bad, f"{kw} step {n}: {bad}"


def _with_map_factors(case, seed=7, amp=0.02):
    """Seeded non-unit map factors on every staggering (the periodic wrap
    face / row repeats face / row 0)."""
    rng = np.random.default_rng(seed)
    m = case.metrics
    for k in ("msftx", "msfty", "msfux", "msfuy", "msfvx", "msfvy"):
        a = 1.0 + amp * rng.standard_normal(getattr(m, k).shape)
        if k in ("msfux", "msfuy"):
            a[:, -1] = a[:, 0]
        if k in ("msfvx", "msfvy"):
            a[-1, :] = a[0, :]
        setattr(m, k, a)
    return case


@pytest.mark.parametrize("top_lid", [False, True])
def test_per_step_parity_rhs_ph_order6_specified(cuda_ready, top_lid):
    """h_sca_adv_order 5 under specified lateral BCs: rhs_ph's order<=6
    horizontal phi advection with its 4th/2nd-order edge rows and the open-top
    face row, on non-unit map factors."""
    case = _with_map_factors(cases.real_like_moist(24, 20, 14, hmax=800.0, specified=True))
    case.controls["h_sca_adv_order"] = 5
    case.controls["top_lid"] = top_lid
    for n, e in enumerate(_per_step(case, 2)):
        bad = {k: v for k, v in e.items() if not v <= _tol(k)}
        assert not bad, f"top_lid={top_lid} step {n}: {bad}"


@pytest.mark.parametrize("shape,theta_opt,moist_opt", [((40, 18, 12), 0, 1), ((18, 40, 12), 2, 2)])
def test_per_step_parity_specified_adv_degrade(cuda_ready, shape, theta_opt, moist_opt):
    """specified_adv_degrade: tiered flux orders near the specified edges and
    no horizontal advection of the outermost cells in the scalar (plain and
    limited), u, v and w operators; grids wider than one 32 x 8 tile so the
    domain edges and the tile edges differ."""
    nx, ny, nz = shape
    case = _with_map_factors(cases.real_like_moist(nx, ny, nz, hmax=800.0, specified=True), seed=5)
    case.controls.update(specified_adv_degrade=True, scalar_adv_opt=theta_opt, moist_adv_opt=moist_opt)
    for n, e in enumerate(_per_step(case, 2)):
        bad = {k: v for k, v in e.items() if not v <= _tol(k)}
        assert not bad, f"{shape} step {n}: {bad}"


@pytest.mark.parametrize("degrade", [False, True])
def test_per_step_parity_specified_bdy_cadence(cuda_ready, degrade):
    """specified_bdy_cadence: relax_bdy_dry tendencies in the relax zone, the
    ring-0 pins of the tangential winds, mu, theta and ph, and the
    zero-gradient w, with perturbed boundary leaves that drift in time and
    non-unit map factors (alone and with the advection degradation)."""
    case = _with_map_factors(cases.real_like_moist(40, 24, 12, hmax=800.0, specified=True, bdy_noise=True), seed=9)
    case.controls.update(specified_bdy_cadence=True, specified_adv_degrade=degrade)
    for n, e in enumerate(_per_step(case, 2)):
        bad = {k: v for k, v in e.items() if not v <= _tol(k)}
        assert not bad, f"degrade={degrade} step {n}: {bad}"


@pytest.mark.parametrize("forcings", [
    dict(nested_ph_relax=True, nested_ph_spec=True),
    dict(nested_ph_relax=True, nested_w_relax=True, nested_ph_spec=True),
    dict(specified_adv_degrade=True, specified_bdy_cadence=True),
])
def test_per_step_parity_nested(cuda_ready, forcings):
    """The nested child (force_geopotential off): the relax-zone ph' / w
    tendencies from the stage state and the ring-0 ph' pin every substep,
    with drifting perturbed leaves and non-unit map factors; and a child
    without forcings, whose specified-only degradation and cadence flags are
    ignored."""
    case = _with_map_factors(cases.real_like_moist(40, 24, 12, hmax=800.0, specified=True, bdy_noise=True), seed=5)
    case.controls.update(force_geopotential=False, **forcings)
    for n, e in enumerate(_per_step(case, 2)):
        bad = {k: v for k, v in e.items() if not v <= _tol(k)}
        assert not bad, f"{forcings} step {n}: {bad}"


@pytest.mark.parametrize("kind,leaves", [
    ("periodic", "all"), ("specified", "all"), ("specified", "saves_only"), ("cadence", "all")])
def test_per_step_parity_physics_tendencies(cuda_ready, kind, leaves):
    """rk_addtend_dry: a DryPhysicsTendencies bundle merged into every stage
    (the boundary saves at the first stage only; h_diabatic coupled by the
    stage mass), with non-unit map factors; a bundle of saves only leaves the
    tendf lanes at zero."""
    from tests.test_oracle_physics_merge import physics_bundle
    specified = kind != "periodic"
    case = _with_map_factors(cases.real_like_moist(28, 22, 12, hmax=800.0, specified=specified,
                                                   bdy_noise=specified), seed=21)
    if kind == "cadence":
        case.controls.update(specified_bdy_cadence=True)
    nz, ny, nx = case.state.theta.shape
    phys = physics_bundle(nz, ny, nx, 17)
    if leaves == "saves_only":
        for f in ("ru_tendf", "rv_tendf", "rw_tendf", "t_tendf", "mu_tendf", "h_diabatic"):
            setattr(phys, f, None)
    for n, e in enumerate(_per_step(case, 2, phys)):
        bad = {k: v for k, v in e.items() if not v <= _tol(k)}
        assert not bad, f"{kind}/{leaves} step {n}: {bad}"


@pytest.mark.parametrize("nx,ny,nz,specified", [(5, 3, 4, False), (33, 9, 7, False), (1, 6, 5, False),
                                                 (7, 7, 5, True)])
def test_per_step_parity_edge_shapes(cuda_ready, nx, ny, nz, specified):
    """Grids smaller than one tile or column block, widths off every tile
    multiple, the minimum 4 levels, a one-column-wide periodic slab and the
    smallest specified domain that holds the five-row boundary strips."""
    case = cases.real_like_moist(nx, ny, nz, hmax=300.0, specified=specified)
    for n, e in enumerate(_per_step(case, 2)):
        bad = {k: v for k, v in e.items() if not v <= _tol(k)}
        assert not bad, f"{(nx, ny, nz, specified)} step {n}: {bad}"


def test_per_step_parity_map_factors_periodic(cuda_ready):
    case = _with_map_factors(cases.real_like_moist(24, 20, 14, hmax=800.0, specified=False), seed=11)
    for n, e in enumerate(_per_step(case, 2)):
        bad = {k: v for k, v in e.items() if not v <= _tol(k)}
        assert not bad, f"step {n}: {bad}"


def test_per_step_parity_warm_bubble_3d(cuda_ready):
    case = cases.warm_bubble_3d(20, 16, 12)
    errs = _per_step(case, 3)
    for n, e in enumerate(errs):
        # u, v, w start at rest: their step-1..3 magnitudes are 1e-3..1e-1 m/s,
        # where one-ulp pow() differences are ~1e-12 relative.
        bad = {k: v for k, v in e.items() if not v <= (1.0e-10 if k in ("u", "v", "w", "u_save", "v_save", "w_save",
                                                                          "mudf", "muave", "ww", "ww_save",
                                                                          "ph_tend", "p_perturbation") else _tol(k))}
        assert not bad, f"step {n}: {bad}"


def test_warm_bubble_2d_500s_reference_gates(cuda_ready):
    """The reference's idealized gate (ic_generators/idealized.py:751-773) on
    the CUDA path: 5000 steps of the 2-D warm bubble, checked against the
    gates, the oracle's own 500 s values and the reference's recorded values."""
    import json
    import os

    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "warm_bubble_2d_500s.json")))
    case = cases.warm_bubble_2d()
    nl = dycore.OperationalNamelist.from_case(case)
    stp = dycore.Stepper(nl)
    a = dycore.carry_from_case(case)
    b = stp.alloc_carry(a)
    for i in range(5000):
        stp.step_into(a, b, lead_seconds=i * nl.dt_s)
        a, b = b, a
    torch.cuda.synchronize()
    x_m, z_m = case.notes["x_m"], case.notes["z_m"]

    def diag(s):
        tp = s.theta.cpu().numpy()[:, 0, :] - 300.0
        wf = s.w.cpu().numpy()[:, 0, :]
        wm = 0.5 * (wf[:-1] + wf[1:])
        wp = np.maximum(tp, 0.0)
        return tp.max(), np.abs(wm).max(), float(np.sum(wp * z_m[:, None]) / wp.sum()), \
            float(np.sum(wp * x_m[None, :]) / wp.sum()), float(s.mu_total.sum().item())

    s0 = dycore.State.from_host(case.state)
    _, _, cz0, _, m0 = diag(s0)
    thmax, wmax, cz, cx, m = diag(a.state)
    rise = cz - cz0
    assert 0.5 <= thmax <= 2.5 and 1.0 <= wmax <= 30.0 and rise >= 500.0 and abs(cx - 10000.0) <= 250.0
    assert abs(m - m0) / m0 <= 1.0e-8
    # the chaotic 5000-step integration amplifies ulp differences, so compare
    # with the oracle's trajectory at the level the reference's own versions
    # agree with each other (~1e-6 relative)
    assert abs(wmax - g["max_abs_w"]) / g["max_abs_w"] < 1.0e-6
    assert abs(rise - g["thermal_rise"]) / g["thermal_rise"] < 1.0e-6
    ref = g["reference_recorded"]
    assert abs(wmax - ref["max_abs_w"]) / ref["max_abs_w"] < 2.0e-4


def test_full_size_properties(cuda_ready):
    """433 x 433 x 50, one step: finite, moisture non-negative under the PD
    limiter; dry mass conserved in the periodic configuration over flat
    terrain.  (Over terrain the reference's edge-padded face averages of mu at
    the domain edge make the periodic mass flux not telescope exactly, and the
    oracle shows the same ~1e-6 drift, so conservation is checked flat.)"""
    case = cases.real_like_moist(433, 433, 50, specified=False)
    nl = dycore.OperationalNamelist.from_case(case)
    carry = dycore.carry_from_case(case)
    out = dycore.rk_scan_step(carry, nl, lead_seconds=0.0)
    torch.cuda.synchronize()
    for f in ("u", "v", "w", "theta", "p_total", "ph_total", "qv"):
        assert torch.isfinite(getattr(out.state, f)).all()
    assert out.state.qv.min().item() >= -1.0e-12
    del out, carry
    flat = cases.real_like_moist(433, 433, 50, hmax=0.0, specified=False)
    nl_f = dycore.OperationalNamelist.from_case(flat)
    carry_f = dycore.carry_from_case(flat)
    out_f = dycore.rk_scan_step(carry_f, nl_f, lead_seconds=0.0)
    torch.cuda.synchronize()
    m0 = carry_f.state.mu_total.sum().item()
    m1 = out_f.state.mu_total.sum().item()
    assert abs(m1 - m0) / m0 < 1.0e-13
    del out_f, carry_f
    # specified configuration on the same grid
    case_s = cases.real_like_moist(433, 433, 50, specified=True)
    nl_s = dycore.OperationalNamelist.from_case(case_s)
    out_s = dycore.rk_scan_step(dycore.carry_from_case(case_s), nl_s, lead_seconds=0.0)
    torch.cuda.synchronize()
    assert torch.isfinite(out_s.state.w).all() and torch.isfinite(out_s.state.theta).all()


@pytest.mark.parametrize("specified,factor,shape", [(False, 0.12, (24, 20, 14)), (True, 0.12, (24, 20, 14)),
                                                    (False, 0.5, (33, 9, 7)), (False, 0.5, (24, 1, 8)),
                                                    (False, 0.5, (24, 2, 8))])
def test_per_step_parity_sixth_order_diffusion(cuda_ready, specified, factor, shape):
    """diff_6th_opt: the monotonic 6th-order filter of u, v, w, theta added to
    every stage's coupled tendencies (operational_mode.py:2870-2876); the
    one-row slab (only v, with its two rows, is filtered along y) and a two-row
    grid exercise the short-axis wrap."""
    case = cases.real_like_moist(*shape, hmax=800.0, specified=specified)
    case.controls.update(diff_6th_opt=2, diff_6th_factor=factor)
    for n, errs in enumerate(_per_step(case, 2 if specified else 3)):
        bad = {k: v for k, v in errs.items() if not v <= _tol(k)}
        assert not bad, f"step {n}: {bad}"


@pytest.mark.parametrize("specified,kw,shape", [
    (False, dict(diff_opt=1, km_opt=4), (24, 20, 14)),
    (True, dict(diff_opt=1, km_opt=4), (24, 20, 14)),
    (False, dict(const_nu_m2_s=75.0), (24, 20, 14)),
    (True, dict(const_nu_m2_s=75.0, diff_opt=1, km_opt=4, diff_6th_opt=2), (33, 9, 7)),
    (False, dict(diff_opt=1, km_opt=4, c_s=0.5), (5, 1, 6)),
])
def test_per_step_parity_explicit_diffusion(cuda_ready, specified, kw, shape):
    """The stage's second-order closures (operational_mode.py:2878-2960): the
    2-D Smagorinsky horizontal diffusion (diff_opt=1, km_opt=4) and the
    constant-K flux form (const_nu_m2_s), alone and together with the
    6th-order filter, on a one-row slab too."""
    case = cases.real_like_moist(*shape, hmax=800.0, specified=specified)
    case.controls.update(kw)
    for n, errs in enumerate(_per_step(case, 2)):
        bad = {k: v for k, v in errs.items() if not v <= _tol(k)}
        assert not bad, f"{kw} step {n}: {bad}"
