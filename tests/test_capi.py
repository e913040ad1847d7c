"""C ABI and host-logic tests that need no GPU: the library loads, exports
every entry point declared in include/wrfgpu.h, and rejects unsupported
configurations before touching the device (the reference raises at trace
time for these, e.g. core/calc_p_rho.py:119-122)."""

from __future__ import annotations

import ctypes
import os
import re

import pytest

from wrf_gpu_b200 import _capi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _capi.load()


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "wrfgpu.h")).read()
    return sorted(set(re.findall(r"\b(wrfgpu_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(lib):
    names = _declared_functions()
    assert "wrfgpu_rk3_step" in names
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_capi.EXPORTED)


def test_params_init_defaults_match_reference_namelist(lib):
    p = _capi.StepParams()
    assert lib.wrfgpu_step_params_init(ctypes.byref(p)) == 0
    # OperationalNamelist defaults (runtime/operational_mode.py:410-700)
    assert p.dt == 10.0 and p.acoustic_substeps == 10 and p.epssm == 0.1
    assert p.top_lid == 0 and p.w_damping == 0 and p.damp_opt == 0 and p.zdamp == 5000.0
    assert p.hypsometric_opt == 1 and p.h_sca_adv_order == 2
    assert p.scalar_adv_opt == 0 and p.moist_adv_opt == 0
    assert p.spec_zone == 1 and p.relax_zone == 4 and p.update_cadence_s == 3600.0
    assert p.moist_cqw == 1 and p.w_coriolis == 1


def _params(lib, **kw):
    p = _capi.StepParams()
    lib.wrfgpu_step_params_init(ctypes.byref(p))
    p.nx, p.ny, p.nz, p.dx, p.dy = 16, 12, 10, 1000.0, 1000.0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("kw,code", [
    (dict(nz=3), _capi.WRFGPU_ERR_BAD_SHAPE),
    (dict(nx=0), _capi.WRFGPU_ERR_BAD_SHAPE),
    (dict(dx=0.0), _capi.WRFGPU_ERR_BAD_SHAPE),
    (dict(hypsometric_opt=3), _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG),
    (dict(scalar_adv_opt=3), _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG),
    (dict(moist_adv_opt=4), _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG),
    (dict(run_boundary=1, relax_zone=6), _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG),
    (dict(precision=7), _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG),
    (dict(column_lanes=7), _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG),
    (dict(column_width=24), _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG),
    (dict(specified_adv_degrade=2), _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG),
    (dict(run_boundary=1, bc_ideal=0, specified_adv_degrade=1, nx=6), _capi.WRFGPU_ERR_BAD_SHAPE),
    (dict(march_levels=7), _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG),
])
def test_validate_rejects(lib, kw, code):
    p = _params(lib, **kw)
    assert lib.wrfgpu_step_params_validate(ctypes.byref(p)) == code
    assert lib.wrfgpu_last_error_string().decode() != ""


def test_validate_accepts_reference_defaults(lib):
    p = _params(lib)
    assert lib.wrfgpu_step_params_validate(ctypes.byref(p)) == 0


def test_batched_rejects_bad_members_before_any_launch(lib):
    p = _params(lib)
    P = (_capi.StepParams * 2)(_params(lib, nz=2), p)
    M = (_capi.Metrics * 2)()
    I = (_capi.StepInputs * 2)()
    O = (_capi.StepOutputs * 2)()
    L = (ctypes.c_double * 2)(0.0, 0.0)
    W = (ctypes.c_void_p * 2)(None, None)
    B = (ctypes.c_size_t * 2)(0, 0)
    assert lib.wrfgpu_rk3_step_batched(2, P, M, I, O, L, W, B, None) == _capi.WRFGPU_ERR_BAD_SHAPE
    P2 = (_capi.StepParams * 2)(p, p)
    assert lib.wrfgpu_rk3_step_batched(2, P2, M, I, O, L, W, B, None) == _capi.WRFGPU_ERR_WORKSPACE
    assert lib.wrfgpu_rk3_step_batched(-1, P, M, I, O, L, W, B, None) == _capi.WRFGPU_ERR_BAD_SHAPE
    assert lib.wrfgpu_rk3_step_batched(0, P, M, I, O, L, W, B, None) == 0


def test_validate_accepts_mixed_precision(lib):
    p = _params(lib, precision=_capi.WRFGPU_PRECISION_MIXED)
    assert lib.wrfgpu_step_params_validate(ctypes.byref(p)) == 0


def test_workspace_size_grows_with_grid_and_options(lib):
    sizes = []
    for kw in (dict(), dict(nx=32), dict(moist_adv_opt=1), dict(run_boundary=1, bc_ideal=0)):
        p = _params(lib, **kw)
        n = ctypes.c_size_t(0)
        assert lib.wrfgpu_step_workspace_size(ctypes.byref(p), ctypes.byref(n)) == 0
        sizes.append(n.value)
    assert sizes[0] > 0 and sizes[1] > sizes[0] and sizes[2] > sizes[0] and sizes[3] > sizes[0]


def test_launch_count(lib):
    p = _params(lib, acoustic_substeps=6)
    n = ctypes.c_int(0)
    assert lib.wrfgpu_step_launch_count(ctypes.byref(p), ctypes.byref(n)) == 0
    # map-factor reciprocals + 3 stages x (8 stage + 3 finish)
    # + 3 launches per substep x (1 + 3 + 6)
    assert n.value == 1 + 3 * 11 + 3 * 10
    # limited moisture: one scale pass over the six species and six tendency
    # passes in the final stage
    for opt in (1, 2):
        p = _params(lib, acoustic_substeps=6, moist_adv_opt=opt)
        assert lib.wrfgpu_step_launch_count(ctypes.byref(p), ctypes.byref(n)) == 0
        assert n.value == 1 + 3 * 11 + 3 * 10 + 7
    # specified boundaries (+2 target launches per stage) with the boundary
    # cadence: + the first stage's mu tendency, one relax launch per stage and
    # one zero-gradient w launch per substep
    p = _params(lib, acoustic_substeps=6, run_boundary=1, bc_ideal=0, specified_bdy_cadence=1)
    assert lib.wrfgpu_step_launch_count(ctypes.byref(p), ctypes.byref(n)) == 0
    assert n.value == (1 + 3 * 13 + 3 * 10) + (1 + 3) + 10
    # a nested child (force_geopotential off) ignores the cadence flag; its
    # relax tendencies add one launch per stage, the ring-0 ph' pin none
    p = _params(lib, acoustic_substeps=6, run_boundary=1, bc_ideal=0, specified_bdy_cadence=1,
                force_geopotential=0, nested_ph_relax=1, nested_w_relax=1, nested_ph_spec=1)
    assert lib.wrfgpu_step_launch_count(ctypes.byref(p), ctypes.byref(n)) == 0
    assert n.value == (1 + 3 * 13 + 3 * 10) + 3


def test_launch_count_with_physics(lib):
    n0, n1 = ctypes.c_int(0), ctypes.c_int(0)
    assert lib.wrfgpu_step_launch_count(ctypes.byref(_params(lib, acoustic_substeps=6)), ctypes.byref(n0)) == 0
    assert lib.wrfgpu_step_launch_count(ctypes.byref(_params(lib, acoustic_substeps=6, physics=1)),
                                        ctypes.byref(n1)) == 0
    # the mu tendency once per step, the u / v / theta merge once per stage
    assert n1.value == n0.value + 1 + 3
    assert lib.wrfgpu_step_params_validate(ctypes.byref(_params(lib, physics=2))) == _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG


def test_params_init_keeps_the_geopotential_forced(lib):
    # BoundaryConfig defaults: force_geopotential on, the nested forcings off
    # (coupling/boundary_apply.py:110, 142-144)
    p = _capi.StepParams()
    lib.wrfgpu_step_params_init(ctypes.byref(p))
    assert p.force_geopotential == 1
    assert p.nested_ph_relax == 0 and p.nested_w_relax == 0 and p.nested_ph_spec == 0


def test_null_pointers_rejected_before_any_launch(lib):
    p = _params(lib)
    m = _capi.Metrics()
    ins = _capi.StepInputs()
    outs = _capi.StepOutputs()
    rc = lib.wrfgpu_rk3_step(ctypes.byref(p), ctypes.byref(m), ctypes.byref(ins), ctypes.byref(outs),
                             float("nan"), None, 0, None)
    assert rc in (_capi.WRFGPU_ERR_WORKSPACE, _capi.WRFGPU_ERR_NULL_POINTER)
    assert lib.wrfgpu_rk3_step(None, None, None, None, 0.0, None, 0, None) == _capi.WRFGPU_ERR_NULL_POINTER


def test_host_shim_rejects_unsupported_namelist():
    import numpy as np
    import torch

    from wrf_gpu_b200 import cases, dycore

    case = cases.warm_bubble_3d(8, 6, 6)
    m = dycore.DycoreMetrics(**{n: torch.as_tensor(np.asarray(getattr(case.metrics, n)))
                                for n in _capi.METRIC_FIELDS},
                             cf1=case.metrics.cf1, cf2=case.metrics.cf2, cf3=case.metrics.cf3,
                             p_top=case.metrics.p_top)
    st = dycore.State.from_host(case.state, device="cpu")
    carry = dycore.initial_operational_carry(st)
    for kw in (dict(use_flux_advection=False), dict(diff_opt=2, km_opt=2), dict(diff_opt=2, km_opt=5),
               dict(const_nu_m2_s=75.0, use_deformation_momentum_diffusion=True),
               dict(acoustic_precision_mode="mixed_perturb_fp32")):
        nl = dycore.OperationalNamelist.from_case(case, metrics=m, **kw)
        with pytest.raises(NotImplementedError):
            dycore.rk_scan_step(carry, nl)


def test_acoustic_substep_rejects_before_any_launch(lib):
    m, c, x = _capi.Metrics(), _capi.AcousticConsts(), _capi.AcousticWork()
    for kw, code in ((dict(run_boundary=1), _capi.WRFGPU_ERR_NULL_POINTER),
                     (dict(w_damping=1), _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG),
                     (dict(), _capi.WRFGPU_ERR_NULL_POINTER)):
        p = _params(lib, **kw)
        assert lib.wrfgpu_acoustic_substep(ctypes.byref(p), ctypes.byref(m), ctypes.byref(c), ctypes.byref(x), 1.0,
                                           None, 0, None) == code
        assert lib.wrfgpu_acoustic_substep_vjp(ctypes.byref(p), ctypes.byref(m), ctypes.byref(c), ctypes.byref(x),
                                               None, ctypes.byref(x), ctypes.byref(x), None, 1.0, None, 0,
                                               None) == code
    n = ctypes.c_size_t(0)
    assert lib.wrfgpu_acoustic_workspace_size(ctypes.byref(_params(lib)), ctypes.byref(n)) == 0 and n.value > 0


def test_lateral_boundary_pass_rejects_before_any_launch(lib):
    ins, outs, lv = _capi.StepInputs(), _capi.StepOutputs(), _capi.LbcLeaves()
    assert lib.wrfgpu_apply_lateral_boundaries(ctypes.byref(_params(lib)), ctypes.byref(ins), ctypes.byref(lv),
                                               ctypes.byref(outs), 0.0, 0, None) == _capi.WRFGPU_ERR_NULL_POINTER
    assert lib.wrfgpu_apply_lateral_boundaries(ctypes.byref(_params(lib)), ctypes.byref(ins), ctypes.byref(lv),
                                               ctypes.byref(outs), float("nan"), 0,
                                               None) == _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG
    assert lib.wrfgpu_apply_lateral_boundaries(None, None, None, None, 0.0, 0, None) == _capi.WRFGPU_ERR_NULL_POINTER


def test_step_epilogue_rejects_before_any_launch(lib):
    p = _params(lib)
    n = ctypes.c_size_t(0)
    assert lib.wrfgpu_step_epilogue_workspace_size(ctypes.byref(p), ctypes.byref(n)) == 0 and n.value > 0
    ins, org, outs = _capi.StepInputs(), _capi.StepInputs(), _capi.StepOutputs()
    assert lib.wrfgpu_step_epilogue(None, None, None, None, None, 0.0, 0, None, None, 0,
                                    None) == _capi.WRFGPU_ERR_NULL_POINTER
    assert lib.wrfgpu_step_epilogue(ctypes.byref(p), ctypes.byref(org), ctypes.byref(ins), None, ctypes.byref(outs),
                                    0.0, 0, None, None, 0, None) == _capi.WRFGPU_ERR_NULL_POINTER


def test_sixth_order_diffusion_params(lib):
    p = _capi.StepParams()
    lib.wrfgpu_step_params_init(ctypes.byref(p))
    assert p.diff_6th_opt == 0 and p.diff_6th_factor == 0.12  # operational_mode.py:491-492
    n0, n1 = ctypes.c_int(0), ctypes.c_int(0)
    assert lib.wrfgpu_step_launch_count(ctypes.byref(_params(lib)), ctypes.byref(n0)) == 0
    assert lib.wrfgpu_step_launch_count(ctypes.byref(_params(lib, diff_6th_opt=2)), ctypes.byref(n1)) == 0
    assert n1.value == n0.value + 3  # one filter launch per stage
    # any nonzero diff_6th_opt switches the filter on, as the reference's int(opt) != 0
    for opt in (3, -1):
        assert lib.wrfgpu_step_params_validate(ctypes.byref(_params(lib, diff_6th_opt=opt))) == 0
        assert lib.wrfgpu_step_launch_count(ctypes.byref(_params(lib, diff_6th_opt=opt)), ctypes.byref(n1)) == 0
        assert n1.value == n0.value + 3
    assert lib.wrfgpu_step_params_validate(ctypes.byref(_params(lib, diff_6th_opt=1, diff_6th_factor=float("nan")))) \
        == _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG


def test_torch_op_is_registered_with_a_fake_implementation():
    """torch.ops.wrfgpu.rk3_step exists and propagates shapes on meta tensors
    (its fake implementation): 16 state leaves, then the 13 carry outputs."""
    import torch

    from wrf_gpu_b200 import torch_ops

    nz, ny, nx = 5, 4, 6
    m = lambda *s: torch.empty(*s, dtype=torch.float64, device="meta")
    shapes = dict(u=(nz, ny, nx + 1), v=(nz, ny + 1, nx), w=(nz + 1, ny, nx), ph_total=(nz + 1, ny, nx),
                  ph_perturbation=(nz + 1, ny, nx), mu_total=(ny, nx), mu_perturbation=(ny, nx))
    fields = [m(*shapes.get(n, (nz, ny, nx))) for n in torch_ops.STEP_FIELDS]
    res = torch.ops.wrfgpu.rk3_step(fields, [], fields[8], None, 0)
    assert len(res) == len(torch_ops.STEP_FIELDS) + len(torch_ops.CARRY_OUT)
    for f, r in zip(fields, res):
        assert r.shape == f.shape and r.dtype == torch.float64
    carry = dict(zip(torch_ops.CARRY_OUT, res[len(fields):]))
    assert carry["ww"].shape == (nz + 1, ny, nx) and carry["mudf"].shape == (ny, nx)
    assert carry["u_save"].shape == (nz, ny, nx + 1)


def test_diffusion_closure_params(lib):
    """diff_opt / km_opt / c_s / const_nu_m2_s: defaults are the reference's,
    the built closures validate and add their launches, the TKE / 3-D
    Smagorinsky pairs are rejected before any launch."""
    p = _capi.StepParams()
    lib.wrfgpu_step_params_init(ctypes.byref(p))
    assert (p.diff_opt, p.km_opt, p.c_s, p.const_nu_m2_s) == (0, 0, 0.25, 0.0)
    p.nx, p.ny, p.nz, p.dx, p.dy, p.dt = 16, 12, 8, 1000.0, 1000.0, 6.0
    base = ctypes.c_int(0)
    assert lib.wrfgpu_step_launch_count(ctypes.byref(p), ctypes.byref(base)) == 0
    ws0 = ctypes.c_size_t(0)
    assert lib.wrfgpu_step_workspace_size(ctypes.byref(p), ctypes.byref(ws0)) == 0
    for kw, extra in ((dict(diff_opt=1, km_opt=4), 2 * 3), (dict(const_nu_m2_s=75.0), 3 * 3),
                      (dict(diff_opt=1, km_opt=4, const_nu_m2_s=75.0), 5 * 3), (dict(diff_opt=1, km_opt=1), 0),
                      (dict(diff_opt=2, km_opt=1), 0)):
        q = _capi.StepParams.from_buffer_copy(p)
        for k, v in kw.items():
            setattr(q, k, v)
        assert lib.wrfgpu_step_params_validate(ctypes.byref(q)) == 0, kw
        n = ctypes.c_int(0)
        assert lib.wrfgpu_step_launch_count(ctypes.byref(q), ctypes.byref(n)) == 0
        assert n.value == base.value + extra, kw
        ws = ctypes.c_size_t(0)
        assert lib.wrfgpu_step_workspace_size(ctypes.byref(q), ctypes.byref(ws)) == 0
        assert (ws.value > ws0.value) == (extra > 0), kw
    for km in (2, 3, 5):
        q = _capi.StepParams.from_buffer_copy(p)
        q.diff_opt, q.km_opt = 2, km
        assert lib.wrfgpu_step_params_validate(ctypes.byref(q)) == _capi.WRFGPU_ERR_UNSUPPORTED_CONFIG
