"""ctypes binding of the C ABI declared in ``include/wrfgpu.h``.

The shared library ``libwrfgpu.so`` is built in-tree by ``wrf_gpu_b200.build``.
Loading fails loudly (``RuntimeError``) when it is missing: there is no CPU
fallback for the step.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libwrfgpu.so"

WRFGPU_OK = 0
WRFGPU_ERR_UNSUPPORTED_CONFIG = 1
WRFGPU_ERR_BAD_SHAPE = 2
WRFGPU_ERR_CUDA = 3
WRFGPU_ERR_NULL_POINTER = 4
WRFGPU_ERR_WORKSPACE = 5
WRFGPU_PRECISION_FP64 = 0
WRFGPU_PRECISION_MIXED = 1
WRFGPU_STATIC_WORKSPACE_BYTES = 32 << 20  # include/wrfgpu.h

_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int


class StepParams(ctypes.Structure):
    _fields_ = [
        ("nx", _I), ("ny", _I), ("nz", _I),
        ("dx", _D), ("dy", _D), ("dt", _D),
        ("acoustic_substeps", _I), ("epssm", _D), ("top_lid", _I), ("w_damping", _I), ("damp_opt", _I),
        ("dampcoef", _D), ("zdamp", _D),
        ("hypsometric_opt", _I), ("h_sca_adv_order", _I), ("scalar_adv_opt", _I), ("moist_adv_opt", _I),
        ("run_boundary", _I), ("bc_ideal", _I), ("spec_zone", _I), ("relax_zone", _I),
        ("update_cadence_s", _D), ("normal_bdy_relax_strength", _D),
        ("moist_cqw", _I), ("w_coriolis", _I), ("precision", _I),
        ("cf1", _D), ("cf2", _D), ("cf3", _D), ("p_top", _D),
        ("cfn", _D), ("cfn1", _D),
        ("march_levels", _I), ("column_lanes", _I), ("column_width", _I), ("specified_adv_degrade", _I),
        ("specified_bdy_cadence", _I), ("force_geopotential", _I), ("nested_ph_relax", _I),
        ("nested_w_relax", _I), ("nested_ph_spec", _I), ("physics", _I),
        ("diff_6th_opt", _I), ("diff_6th_factor", _D),
        ("diff_opt", _I), ("km_opt", _I), ("c_s", _D), ("const_nu_m2_s", _D),
    ]


METRIC_FIELDS = ("c1h", "c2h", "c3h", "c4h", "c1f", "c2f", "c3f", "c4f", "dn", "dnw", "rdn", "rdnw", "fnm", "fnp",
                 "msftx", "msfty", "msfux", "msfuy", "msfvx", "msfvy", "f", "e", "sina", "cosa")


class Metrics(ctypes.Structure):
    _fields_ = [(n, _P) for n in METRIC_FIELDS]


STATE_FIELDS = ("u", "v", "w", "theta", "p_total", "p_perturbation", "ph_total", "ph_perturbation",
                "mu_total", "mu_perturbation")


# DryPhysicsTendencies leaves (dynamics/core/rk_addtend_dry.py:103-124) and their C input names
PHYSICS_LEAVES = ("ru_tendf", "rv_tendf", "rw_tendf", "ph_tendf", "t_tendf", "mu_tendf", "h_diabatic", "u_save",
                  "v_save", "w_save", "ph_save", "t_save")
PHYSICS_FIELDS = ("ru_tendf", "rv_tendf", "rw_tendf", "ph_tendf", "t_tendf", "mu_tendf", "h_diabatic", "phys_u_save",
                  "phys_v_save", "phys_w_save", "phys_ph_save", "phys_t_save")


class StepInputs(ctypes.Structure):
    _fields_ = [(n, _P) for n in STATE_FIELDS] + [
        ("q", _P * 6), ("mudf", _P),
        ("base_u", _P), ("base_v", _P), ("base_w", _P), ("base_theta", _P), ("base_mu", _P),
        ("u_bdy", _P), ("v_bdy", _P), ("bdy_ntime", _I), ("bdy_width", _I), ("bdy_side_len", _I),
        ("theta_bdy", _P), ("ph_bdy", _P), ("mu_bdy", _P), ("w_bdy", _P),
    ] + [(n, _P) for n in PHYSICS_FIELDS]


CARRY_OUT_FIELDS = ("t_2ave", "ww", "mudf", "muave", "muts", "ph_tend", "u_save", "v_save", "w_save", "t_save",
                    "ph_save", "mu_save", "ww_save")


class StepOutputs(ctypes.Structure):
    _fields_ = [(n, _P) for n in STATE_FIELDS] + [("q", _P * 6)] + [(n, _P) for n in CARRY_OUT_FIELDS]


ACOUSTIC_WORK_FIELDS = ("u", "v", "w", "ph", "theta_w", "t_2ave", "p", "pm1", "al", "ww", "mu", "muts", "muave",
                        "mudf")
ACOUSTIC_CONST_FIELDS = ("u_tend", "v_tend", "t_tend", "rw_tend", "ph_tend", "alt", "pb", "c2a", "cqu", "cqv", "cqw",
                         "php", "pt1", "a", "alpha", "gamma", "ww_1", "mut", "muu", "muv", "mu_tend", "u_1", "v_1",
                         "w_save", "theta", "phb0", "u_target", "v_target")


class AcousticWork(ctypes.Structure):
    _fields_ = [(n, _P) for n in ACOUSTIC_WORK_FIELDS]


class AcousticConsts(ctypes.Structure):
    _fields_ = [(n, _P) for n in ACOUSTIC_CONST_FIELDS]


ACOUSTIC_TEND_FIELDS = ("u_tend", "v_tend", "t_tend", "rw_tend", "ph_tend", "mu_tend")


class AcousticTendCot(ctypes.Structure):
    _fields_ = [(n, _P) for n in ACOUSTIC_TEND_FIELDS]


class LbcLeaves(ctypes.Structure):
    _fields_ = [("u", _P), ("v", _P), ("w", _P), ("theta", _P), ("q", _P * 6), ("p", _P), ("pb", _P), ("mu", _P),
                ("mub", _P), ("ph", _P), ("phb", _P), ("ntime", _I), ("width", _I), ("side_len", _I)]


class NestInterp(ctypes.Structure):
    _fields_ = [("y0", _P), ("y1", _P), ("x0", _P), ("x1", _P), ("wy", _P), ("wx", _P), ("child_ny", _I),
                ("child_nx", _I), ("parent_ny", _I), ("parent_nx", _I)]


class NestFeedbackPlan(ctypes.Structure):
    _fields_ = [("parent_lin", _P), ("child_lin", _P), ("npts", _I), ("stencil", _I), ("pwe", _I), ("psn", _I),
                ("cwe", _I), ("csn", _I), ("i_lo", _I), ("i_hi", _I), ("j_lo", _I), ("j_hi", _I), ("smooth", _I)]


class RowBlock(ctypes.Structure):
    """``wrfgpu_row_block``: rows [row0, row0 + nrows) of a (nz, ny, nx) array,
    packed at element ``offset`` of a buffer."""
    _fields_ = [("field", _P), ("nz", _I), ("ny", _I), ("nx", _I), ("row0", _I), ("nrows", _I),
                ("offset", ctypes.c_longlong)]


MAX_ROW_BLOCKS = 40


# wrfgpu_theta_limiter_diag: 4 int32 (count, x, y, z) then 3 float64 (mass before, after, residual)
THETA_DIAG_BYTES = 40


EXPORTED = ("wrfgpu_step_params_init", "wrfgpu_step_params_validate", "wrfgpu_step_workspace_size",
            "wrfgpu_rk3_step", "wrfgpu_rk3_step_device_lead", "wrfgpu_rk3_step_static_workspace",
            "wrfgpu_rk3_step_batched", "wrfgpu_autotune", "wrfgpu_scalar_advection",
            "wrfgpu_scalar_advection_adjoint", "wrfgpu_scalar_advection_vjp", "wrfgpu_flux_advection",
            "wrfgpu_flux_advection_vjp", "wrfgpu_w_vertical_advection", "wrfgpu_w_vertical_advection_vjp",
            "wrfgpu_acoustic_workspace_size", "wrfgpu_acoustic_substep",
            "wrfgpu_acoustic_substep_vjp", "wrfgpu_apply_lateral_boundaries",
            "wrfgpu_step_epilogue_workspace_size", "wrfgpu_step_epilogue", "wrfgpu_step_epilogue_device_lead", "wrfgpu_step_launch_count", "wrfgpu_profile_enable", "wrfgpu_profile_read",
            "wrfgpu_profile_class_count", "wrfgpu_profile_class_name", "wrfgpu_last_error_string",
            "wrfgpu_version", "wrfgpu_nest_interp_field", "wrfgpu_nest_ring_leaf", "wrfgpu_nest_feedback",
            "wrfgpu_nest_rebuild_total", "wrfgpu_copy_rows",
            "wrfgpu_rows_pack", "wrfgpu_rows_unpack")

_lib = None


def load(path: str | os.PathLike | None = None):
    """Load ``libwrfgpu.so`` (raises ``RuntimeError`` if it is absent)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"wrf_gpu_b200: CUDA library {p} is missing; build it with "
            "`python -c 'import wrf_gpu_b200.build as b; b.build()'` (there is no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    lib.wrfgpu_step_params_init.argtypes = [ctypes.POINTER(StepParams)]
    lib.wrfgpu_step_params_init.restype = _I
    lib.wrfgpu_step_params_validate.argtypes = [ctypes.POINTER(StepParams)]
    lib.wrfgpu_step_params_validate.restype = _I
    lib.wrfgpu_step_workspace_size.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(ctypes.c_size_t)]
    lib.wrfgpu_step_workspace_size.restype = _I
    lib.wrfgpu_step_launch_count.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(_I)]
    lib.wrfgpu_step_launch_count.restype = _I
    lib.wrfgpu_rk3_step.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics), ctypes.POINTER(StepInputs),
                                    ctypes.POINTER(StepOutputs), _D, _P, ctypes.c_size_t, _P]
    lib.wrfgpu_rk3_step.restype = _I
    lib.wrfgpu_rk3_step_device_lead.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics),
                                                ctypes.POINTER(StepInputs), ctypes.POINTER(StepOutputs), _P, _P,
                                                ctypes.c_size_t, _P]
    lib.wrfgpu_rk3_step_device_lead.restype = _I
    lib.wrfgpu_rk3_step_static_workspace.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics),
                                                     ctypes.POINTER(StepInputs), ctypes.POINTER(StepOutputs), _D, _P]
    lib.wrfgpu_rk3_step_static_workspace.restype = _I
    lib.wrfgpu_rk3_step_batched.argtypes = [_I, ctypes.POINTER(StepParams), ctypes.POINTER(Metrics),
                                            ctypes.POINTER(StepInputs), ctypes.POINTER(StepOutputs),
                                            ctypes.POINTER(_D), ctypes.POINTER(_P), ctypes.POINTER(ctypes.c_size_t), _P]
    lib.wrfgpu_rk3_step_batched.restype = _I
    lib.wrfgpu_autotune.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics), ctypes.POINTER(StepInputs),
                                    ctypes.POINTER(StepOutputs), _P, ctypes.c_size_t, _P]
    lib.wrfgpu_autotune.restype = _I
    for name in ("wrfgpu_scalar_advection", "wrfgpu_scalar_advection_adjoint"):
        fn = getattr(lib, name)
        fn.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics), _P, _P, _P, _P, _P, _P]
        fn.restype = _I
    lib.wrfgpu_scalar_advection_vjp.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics),
                                                _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]
    lib.wrfgpu_scalar_advection_vjp.restype = _I
    lib.wrfgpu_flux_advection.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics),
                                          _P, _P, _P, _P, _P, _P, _P, _P]
    lib.wrfgpu_flux_advection.restype = _I
    lib.wrfgpu_flux_advection_vjp.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics),
                                              _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]
    lib.wrfgpu_flux_advection_vjp.restype = _I
    lib.wrfgpu_w_vertical_advection.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics), _P, _P, _P, _P]
    lib.wrfgpu_w_vertical_advection.restype = _I
    lib.wrfgpu_w_vertical_advection_vjp.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics),
                                                    _P, _P, _P, _P, _P, _P]
    lib.wrfgpu_w_vertical_advection_vjp.restype = _I
    lib.wrfgpu_acoustic_workspace_size.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(ctypes.c_size_t)]
    lib.wrfgpu_acoustic_workspace_size.restype = _I
    lib.wrfgpu_acoustic_substep.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics),
                                            ctypes.POINTER(AcousticConsts), ctypes.POINTER(AcousticWork), _D, _P,
                                            ctypes.c_size_t, _P]
    lib.wrfgpu_acoustic_substep.restype = _I
    lib.wrfgpu_acoustic_substep_vjp.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(Metrics),
                                                ctypes.POINTER(AcousticConsts), ctypes.POINTER(AcousticWork),
                                                ctypes.POINTER(AcousticWork), ctypes.POINTER(AcousticWork),
                                                ctypes.POINTER(AcousticWork), ctypes.POINTER(AcousticTendCot), _D,
                                                _P, ctypes.c_size_t, _P]
    lib.wrfgpu_acoustic_substep_vjp.restype = _I
    lib.wrfgpu_apply_lateral_boundaries.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(StepInputs),
                                                    ctypes.POINTER(LbcLeaves), ctypes.POINTER(StepOutputs), _D, _I,
                                                    _P]
    lib.wrfgpu_apply_lateral_boundaries.restype = _I
    lib.wrfgpu_step_epilogue_workspace_size.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(ctypes.c_size_t)]
    lib.wrfgpu_step_epilogue_workspace_size.restype = _I
    lib.wrfgpu_step_epilogue.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(StepInputs),
                                         ctypes.POINTER(StepInputs), ctypes.POINTER(LbcLeaves),
                                         ctypes.POINTER(StepOutputs), _D, _I, _P, _P, ctypes.c_size_t, _P]
    lib.wrfgpu_step_epilogue.restype = _I
    lib.wrfgpu_step_epilogue_device_lead.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(StepInputs),
                                                     ctypes.POINTER(StepInputs), ctypes.POINTER(LbcLeaves),
                                                     ctypes.POINTER(StepOutputs), _P, _I, _P, _P, ctypes.c_size_t,
                                                     _P]
    lib.wrfgpu_step_epilogue_device_lead.restype = _I
    lib.wrfgpu_nest_interp_field.argtypes = [ctypes.POINTER(NestInterp), _P, _I, _P, _P]
    lib.wrfgpu_nest_interp_field.restype = _I
    lib.wrfgpu_nest_ring_leaf.argtypes = [ctypes.POINTER(NestInterp), _P, _P, _P, _I, _I, _I, _I, _I, _I, _I, _P,
                                          _P]
    lib.wrfgpu_nest_ring_leaf.restype = _I
    lib.wrfgpu_nest_feedback.argtypes = [ctypes.POINTER(NestFeedbackPlan), _P, _P, _I, _P, _P, _P]
    lib.wrfgpu_nest_feedback.restype = _I
    lib.wrfgpu_nest_rebuild_total.argtypes = [_P, _P, _P, ctypes.c_size_t, _P, _P]
    lib.wrfgpu_nest_rebuild_total.restype = _I
    lib.wrfgpu_copy_rows.argtypes = [_P, _I, _I, _I, _P, _I, _I, _I, _I, _P]
    lib.wrfgpu_copy_rows.restype = _I
    for name in ("wrfgpu_rows_pack", "wrfgpu_rows_unpack"):
        getattr(lib, name).argtypes = [ctypes.POINTER(RowBlock), _I, _P, ctypes.c_longlong, _P]
        getattr(lib, name).restype = _I
    lib.wrfgpu_profile_enable.argtypes = [_I, _I]
    lib.wrfgpu_profile_enable.restype = _I
    lib.wrfgpu_profile_read.argtypes = [ctypes.POINTER(_D), ctypes.POINTER(_I), _I, ctypes.POINTER(_I)]
    lib.wrfgpu_profile_read.restype = _I
    lib.wrfgpu_profile_class_count.argtypes = []
    lib.wrfgpu_profile_class_count.restype = _I
    lib.wrfgpu_profile_class_name.argtypes = [_I]
    lib.wrfgpu_profile_class_name.restype = ctypes.c_char_p
    lib.wrfgpu_last_error_string.argtypes = []
    lib.wrfgpu_last_error_string.restype = ctypes.c_char_p
    lib.wrfgpu_version.argtypes = []
    lib.wrfgpu_version.restype = ctypes.c_char_p
    if path is None:
        _lib = lib
    return lib


class WrfGpuError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, code: int, message: str):
        super().__init__(f"wrfgpu error {code}: {message}")
        self.code = code


def check(code: int) -> None:
    if code != WRFGPU_OK:
        raise WrfGpuError(code, load().wrfgpu_last_error_string().decode())


def profile_enable(enable: bool, max_records: int = 8192) -> None:
    check(load().wrfgpu_profile_enable(int(bool(enable)), int(max_records)))


def profile_read() -> dict:
    """Summed device milliseconds and launch counts per kernel class (synchronises)."""
    lib = load()
    n = lib.wrfgpu_profile_class_count()
    ms = (_D * n)()
    cnt = (_I * n)()
    dropped = _I(0)
    check(lib.wrfgpu_profile_read(ms, cnt, n, ctypes.byref(dropped)))
    return {lib.wrfgpu_profile_class_name(c).decode(): (float(ms[c]), int(cnt[c])) for c in range(n)}
