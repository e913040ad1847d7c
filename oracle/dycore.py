"""NumPy float64 restatement of wrf_gpu's RK3 split-explicit dycore step.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Arrays are ``(k, j, i)``
C-order; u lives on ``(nz, ny, nx+1)`` x-faces, v on ``(nz, ny+1, nx)``
y-faces, w/ph on ``(nz+1, ny, nx)`` full levels, 2-D fields are ``(ny, nx)``.
Reference paths below are relative to ``src/gpuwrf``.
"""

from __future__ import annotations

from dataclasses import dataclass, field, replace
from types import SimpleNamespace

import numpy as np

# --- constants: dynamics/acoustic_wrf.py:27-75, core/advance_w.py:28,87-88,
#     runtime/operational_mode.py:202, core/acoustic.py:846-847, calc_p_rho.py:24
R_D = 287.0
CP_D = 7.0 * R_D / 2.0
P0 = 100000.0
CPOVCV = CP_D / (CP_D - R_D)
CVPM = -(CP_D - R_D) / CP_D
G = 9.81
T0 = 300.0
MIN_ACOUSTIC_ALT = 0.1
W_RERADIUS = 1.0 / 6370.0e3
W_ALPHA = 0.3
W_BETA = 1.0
PD_EPS = 1.0e-20
EMDIV = 0.01
SMDIV = 0.1
MIN_MUTS_FRACTION = 0.5
MIN_MUTS_PA = 1.0
NORMAL_BDY_RELAX_STRENGTH = 20.0
MOIST_SPECIES = ("qv", "qc", "qr", "qi", "qs", "qg")
SIDES = ("W", "E", "S", "N")


# ----------------------------------------------------------------------------
# containers
# ----------------------------------------------------------------------------

@dataclass
class Namelist:
    """The ``OperationalNamelist`` fields the step reads (operational_mode.py:410-700)."""

    metrics: SimpleNamespace
    dx: float
    dy: float
    dt_s: float = 10.0
    acoustic_substeps: int = 10
    epssm: float = 0.1
    top_lid: bool = False
    w_damping: int = 0
    damp_opt: int = 0
    dampcoef: float = 0.0
    zdamp: float = 5000.0
    hypsometric_opt: int = 1
    h_sca_adv_order: int = 2
    specified_adv_degrade: bool = False   # operational_mode.py:460 (opt-in)
    specified_bdy_cadence: bool = False   # operational_mode.py:453 (opt-in)
    force_geopotential: bool = True       # BoundaryConfig (boundary_apply.py:110); False = nested child
    nested_ph_relax: bool = False         # boundary_apply.py:142-144 (opt-in nested forcings)
    nested_w_relax: bool = False
    nested_ph_spec: bool = False
    scalar_adv_opt: int = 0
    moist_adv_opt: int = 0
    run_boundary: bool = False
    bc_ideal: bool = True
    spec_zone: int = 1
    relax_zone: int = 4
    update_cadence_s: float = 3600.0
    normal_bdy_relax_strength: float | None = None
    moist_cqw: bool = True          # GPUWRF_MOIST_CQW default (operational_mode.py:219)
    w_coriolis: bool = True         # GPUWRF_W_CORIOLIS default (operational_mode.py:1793)
    diff_6th_opt: int = 0           # operational_mode.py:491 (0 off; 1 and 2 apply the monotonic filter)
    diff_6th_factor: float = 0.12   # operational_mode.py:492
    diff_opt: int = 0               # operational_mode.py:475 (1 with km_opt 4: 2-D Smagorinsky)
    km_opt: int = 0                 # operational_mode.py:476
    c_s: float = 0.25               # operational_mode.py:482 (explicit_diffusion.py:957 C_S_DEFAULT)
    const_nu_m2_s: float = 0.0      # operational_mode.py:494 (> 0: constant-K diffusion)
    base_tend: dict | None = None   # namelist.tendencies u/v/w/theta/mu (zero when None)


def lateral_flags(nl: Namelist):
    """``_acoustic_lateral_bc_flags`` (operational_mode.py:1247-1254): periodic,
    specified, nested; a boundary domain without force_geopotential is nested."""
    if not (nl.run_boundary and not nl.bc_ideal):
        return True, False, False
    nested = not nl.force_geopotential
    return False, not nested, nested


def copy_state(s: SimpleNamespace) -> SimpleNamespace:
    return SimpleNamespace(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in vars(s).items()})


# ----------------------------------------------------------------------------
# small helpers
# ----------------------------------------------------------------------------

def _col(a):
    return np.asarray(a)[:, None, None]


def xpair(f):
    """Edge-padded x-face pair (core/acoustic.py:544-547)."""
    left = np.concatenate([f[..., :1], f], axis=-1)
    right = np.concatenate([f, f[..., -1:]], axis=-1)
    return left, right


def ypair(f):
    """Edge-padded y-face pair (core/acoustic.py:550-553)."""
    south = np.concatenate([f[..., :1, :], f], axis=-2)
    north = np.concatenate([f, f[..., -1:, :]], axis=-2)
    return south, north


def u_face_average_2d(f):
    """core/small_step_prep.py:75-79."""
    return np.concatenate((f[:, :1], 0.5 * (f[:, :-1] + f[:, 1:]), f[:, -1:]), axis=1)


def v_face_average_2d(f):
    """core/small_step_prep.py:82-86."""
    return np.concatenate((f[:1, :], 0.5 * (f[:-1, :] + f[1:, :]), f[-1:, :]), axis=0)


def inv_density(theta, p):
    """dynamics/acoustic_wrf.py:187-206 (qvf = 1)."""
    return (R_D / P0) * theta * 1.0 * ((np.maximum(p, 1.0) / P0) ** CVPM)


def pressure_from_theta_alt(theta, alt):
    """dynamics/acoustic_wrf.py:209-221 (qvf = 1)."""
    argument = (R_D * theta * 1.0) / (P0 * np.maximum(alt, 1.0e-8))
    return P0 * (np.maximum(argument, 1.0e-12) ** CPOVCV)


def qtot_of(s):
    return s.qv + s.qc + s.qr + s.qi + s.qs + s.qg


def moisture_coupling_factors(s):
    """dynamics/acoustic_wrf.py:305-320."""
    qtot = qtot_of(s)
    ql, qr = xpair(qtot)
    qs_, qn = ypair(qtot)
    return 1.0 / (1.0 + 0.5 * (ql + qr)), 1.0 / (1.0 + 0.5 * (qs_ + qn))


# ----------------------------------------------------------------------------
# flux-form advection: dynamics/flux_advection.py
# ----------------------------------------------------------------------------

def flux5_face(f, vel, axis):
    """flux_advection.py:53-88: left-face 5th-order upwind value."""
    q_im3 = np.roll(f, 3, axis=axis)
    q_im2 = np.roll(f, 2, axis=axis)
    q_im1 = np.roll(f, 1, axis=axis)
    q_ip1 = np.roll(f, -1, axis=axis)
    q_ip2 = np.roll(f, -2, axis=axis)
    f6 = (37.0 * (f + q_im1) - 8.0 * (q_ip1 + q_im2) + (q_ip2 + q_im3)) / 60.0
    corr = ((q_ip2 - q_im3) - 5.0 * (q_ip1 - q_im2) + 10.0 * (f - q_im1)) / 60.0
    return f6 - np.sign(vel) * corr


def couple_velocities_periodic(u, v, mu_total, m, rdx, rdy):
    """flux_advection.py:394-470 (calc_ww_cp on periodic collapsed faces)."""
    nz = u.shape[0]
    ny, nx = mu_total.shape
    u_f = u[..., :nx]
    v_f = v[:, :ny, :]
    msfuy = m.msfuy[:, :nx]
    msfvx = m.msfvx[:ny, :]
    muu = 0.5 * (mu_total + np.roll(mu_total, 1, axis=-1))
    muv = 0.5 * (mu_total + np.roll(mu_total, 1, axis=-2))
    mass_u = _col(m.c1h) * muu[None] + _col(m.c2h)
    mass_v = _col(m.c1h) * muv[None] + _col(m.c2h)
    ru = mass_u * u_f / msfuy[None]
    rv = mass_v * v_f / msfvx[None]
    divv = _col(m.dnw) * m.msftx[None] * (rdx * (np.roll(ru, -1, -1) - ru) + rdy * (np.roll(rv, -1, -2) - rv))
    dmdt = np.sum(divv, axis=0, keepdims=True)
    inc = -(_col(m.dnw) * _col(m.c1h) * dmdt) - divv
    cum = np.cumsum(inc, axis=0)
    rom = np.zeros((nz + 1, ny, nx))
    rom[1:nz] = cum[: nz - 1]
    return SimpleNamespace(ru=ru, rv=rv, rom=rom, msftx=m.msftx, msfux=m.msfux[:, :nx],
                           msfvy=m.msfvy[:ny, :], msfvx=msfvx)


def stage_omega_specified(u, v, mu_total, m, rdx, rdy):
    """flux_advection.py:180-232 (edge-faithful calc_ww_cp)."""
    nz = u.shape[0]
    ny, nx = mu_total.shape
    mpx = np.pad(mu_total, ((0, 0), (1, 0)), mode="edge")
    muu = 0.5 * (mpx[:, 1:] + mpx[:, :-1])
    muu = np.concatenate([muu, mu_total[:, -1:]], axis=1)
    mpy = np.pad(mu_total, ((1, 0), (0, 0)), mode="edge")
    muv = 0.5 * (mpy[1:, :] + mpy[:-1, :])
    muv = np.concatenate([muv, mu_total[-1:, :]], axis=0)
    c1 = _col(m.c1h)
    c2 = _col(m.c2h)
    ru = (c1 * muu[None] + c2) * u / m.msfuy[None]
    rv = (c1 * muv[None] + c2) * v / m.msfvx[None]
    divv = m.msftx[None] * _col(m.dnw) * (rdx * (ru[:, :, 1:] - ru[:, :, :-1]) + rdy * (rv[:, 1:, :] - rv[:, :-1, :]))
    dmdt = np.sum(divv, axis=0, keepdims=True)
    inc = -(_col(m.dnw) * _col(m.c1h) * dmdt) - divv
    cum = np.cumsum(inc, axis=0)
    rom = np.zeros((nz + 1, ny, nx))
    rom[1:nz] = cum[: nz - 1]
    return rom


def _shift0(f, k, axis):
    """flux_advection.py:257-278: shift by k along axis (value at i is f[i-k]) with zero fill."""
    n = f.shape[axis]
    out = np.zeros_like(f)
    src = [slice(None)] * f.ndim
    dst = [slice(None)] * f.ndim
    if k >= 0:
        src[axis], dst[axis] = slice(0, n - k), slice(k, n)
    else:
        src[axis], dst[axis] = slice(-k, n), slice(0, n + k)
    out[tuple(dst)] = f[tuple(src)]
    return out


def _axis_idx(f, axis):
    shape = [1] * f.ndim
    shape[axis] = f.shape[axis]
    return np.arange(f.shape[axis]).reshape(shape)


def specified_flux_faces(f, vel, axis, upstream=False):
    """flux_advection.py:288-347: tiered order-5 fluxes under specified BCs.
    Face m (between cells m-1 and m) of an axis of n cells: flux5 on 3..n-3,
    flux3 (+sign(vel) correction) on 2 and n-2, 2nd order on 1 and n-1 (with
    the upstream normal-wind rule when ``upstream``), zero on face 0."""
    q_im3, q_im2, q_im1 = _shift0(f, 3, axis), _shift0(f, 2, axis), _shift0(f, 1, axis)
    q_ip1, q_ip2 = _shift0(f, -1, axis), _shift0(f, -2, axis)
    face6 = (37.0 * (f + q_im1) - 8.0 * (q_ip1 + q_im2) + (q_ip2 + q_im3)) / 60.0
    corr6 = ((q_ip2 - q_im3) - 5.0 * (q_ip1 - q_im2) + 10.0 * (f - q_im1)) / 60.0
    face5 = face6 - np.sign(vel) * corr6
    face4 = (7.0 * (f + q_im1) - (q_ip1 + q_im2)) / 12.0
    corr4 = ((q_ip1 - q_im2) - 3.0 * (f - q_im1)) / 12.0
    face3 = face4 + np.sign(vel) * corr4
    face2 = 0.5 * (f + q_im1)
    n = f.shape[axis]
    idx = _axis_idx(f, axis)
    if upstream:
        low = 0.5 * (f + np.where(f < 0.0, f, q_im1))
        high = 0.5 * (q_im1 + np.where(q_im1 > 0.0, q_im1, f))
        face2 = np.where(idx == 1, low, np.where(idx == n - 1, high, face2))
    five = (idx >= 3) & (idx <= n - 3)
    three = (idx == 2) | (idx == n - 2)
    two = (idx == 1) | (idx == n - 1)
    return vel * np.where(five, face5, np.where(three, face3, np.where(two, face2, 0.0)))


def specified_div(fq, axis):
    """flux_advection.py:350-361: fq(m+1) - fq(m) on cells 1..n-2, zero on the outermost cells."""
    d = _shift0(fq, -1, axis) - fq
    idx = _axis_idx(fq, axis)
    return np.where((idx >= 1) & (idx <= fq.shape[axis] - 2), d, 0.0)


def couple_uv_specified(u, v, mu_total, m):
    """flux_advection.py:364-391: full-face coupled velocities with edge-padded face masses."""
    mpx = np.pad(mu_total, ((0, 0), (1, 0)), mode="edge")
    muu = np.concatenate([0.5 * (mpx[:, 1:] + mpx[:, :-1]), mu_total[:, -1:]], axis=1)
    mpy = np.pad(mu_total, ((1, 0), (0, 0)), mode="edge")
    muv = np.concatenate([0.5 * (mpy[1:, :] + mpy[:-1, :]), mu_total[-1:, :]], axis=0)
    c1, c2 = _col(m.c1h), _col(m.c2h)
    return (c1 * muu[None] + c2) * u / m.msfuy[None], (c1 * muv[None] + c2) * v / m.msfvx[None]


def _vflux_scalar(f, rom, fzm, fzp):
    """flux_advection.py:534-562 / 678-711 (order-3 vertical flux, rigid ends)."""
    nz = f.shape[0]
    vflux = np.zeros((nz + 1,) + f.shape[1:])
    q_km2, q_km1, q_k, q_kp1 = f[: nz - 3], f[1 : nz - 2], f[2 : nz - 1], f[3:nz]
    velz = -rom[2 : nz - 1]
    flux4 = (7.0 * (q_k + q_km1) - (q_kp1 + q_km2)) / 12.0
    corr = ((q_kp1 - q_km2) - 3.0 * (q_k - q_km1)) / 12.0
    vflux[2 : nz - 1] = rom[2 : nz - 1] * (flux4 + np.sign(velz) * corr)
    vflux[1] = rom[1] * (fzm[1] * f[1] + fzp[1] * f[0])
    vflux[nz - 1] = rom[nz - 1] * (fzm[nz - 1] * f[nz - 1] + fzp[nz - 1] * f[nz - 2])
    return vflux


def advect_scalar_flux(f, vel, rdx, rdy, rdzw, fzm, fzp):
    """flux_advection.py:482-568 (h5/v3 periodic)."""
    msftx = vel.msftx[None]
    if getattr(vel, "specified", False):  # :512-520
        tend = -msftx * rdx * specified_div(specified_flux_faces(f, vel.ru, 2), 2)
        tend = tend - msftx * rdy * specified_div(specified_flux_faces(f, vel.rv, 1), 1)
    else:
        fqx = vel.ru * flux5_face(f, vel.ru, 2)
        tend = -msftx * rdx * (np.roll(fqx, -1, 2) - fqx)
        fqy = vel.rv * flux5_face(f, vel.rv, 1)
        tend = tend - msftx * rdy * (np.roll(fqy, -1, 1) - fqy)
    nz = f.shape[0]
    vflux = _vflux_scalar(f, vel.rom, fzm, fzp)
    return tend - _col(rdzw) * (vflux[1:] - vflux[:nz])


def _flux_upwind_face(fo, vel, mu_face, dxy, dt, axis):
    """flux_advection.py:614-641."""
    q_im1 = np.roll(fo, 1, axis=axis)
    cr = vel * dt / dxy / mu_face
    a = np.abs(cr)
    return mu_face * (dxy / dt) * (0.5 * np.minimum(1.0, cr + a) * q_im1 + 0.5 * np.maximum(-1.0, cr - a) * fo)


def _flux_upwind_face_z(fo, rom, mu_h, rdzw, dt):
    """flux_advection.py:644-675."""
    nz = fo.shape[0]
    out = np.zeros((nz + 1,) + fo.shape[1:])
    q_km1, q_k = fo[: nz - 1], fo[1:nz]
    dz = 2.0 / (_col(rdzw[1:nz]) + _col(rdzw[: nz - 1]))
    mu_face = 0.5 * (mu_h[1:nz] + mu_h[: nz - 1])
    cr = rom[1:nz] * dt / dz / mu_face
    a = np.abs(cr)
    out[1:nz] = mu_face * (dz / dt) * (0.5 * np.minimum(1.0, cr + a) * q_km1 + 0.5 * np.maximum(-1.0, cr - a) * q_k)
    return out


def advect_scalar_flux_limited(f, fo, vel, opt, mut, mu_old, m, rdx, rdy, dt):
    """flux_advection.py:736-1000 (PD opt 1 / monotonic opt 2, periodic path)."""
    nz = f.shape[0]
    msftx = vel.msftx[None]
    rdzw = m.rdnw
    c1, c2 = _col(m.c1h), _col(m.c2h)
    mu_h = c1 * mut[None] + c2
    muu = 0.5 * (mut + np.roll(mut, 1, -1))
    muv = 0.5 * (mut + np.roll(mut, 1, -2))
    mu_u = c1 * muu[None] + c2
    mu_v = c1 * muv[None] + c2
    dx, dy = 1.0 / rdx, 1.0 / rdy
    spec = bool(getattr(vel, "specified", False))  # :816-828, 841, 963-968
    ip1 = (lambda a, ax: _shift0(a, -1, ax)) if spec else (lambda a, ax: np.roll(a, -1, ax))
    fqxl = _flux_upwind_face(fo, vel.ru, mu_u, dx, dt, 2)
    fqyl = _flux_upwind_face(fo, vel.rv, mu_v, dy, dt, 1)
    fqzl = _flux_upwind_face_z(fo, vel.rom, mu_h, rdzw, dt)
    if spec:
        fqxl = np.where(_axis_idx(fqxl, 2) == 0, 0.0, fqxl)
        fqyl = np.where(_axis_idx(fqyl, 1) == 0, 0.0, fqyl)
        fqx = specified_flux_faces(f, vel.ru, 2) - fqxl
        fqy = specified_flux_faces(f, vel.rv, 1) - fqyl
    else:
        fqx = vel.ru * flux5_face(f, vel.ru, 2) - fqxl
        fqy = vel.rv * flux5_face(f, vel.rv, 1) - fqyl
    fqz = _vflux_scalar(f, vel.rom, m.fnm, m.fnp) - fqzl
    mass_old = c1 * mu_old[None] + c2
    div_low = (msftx * msftx * (rdx * (ip1(fqxl, 2) - fqxl) + rdy * (ip1(fqyl, 1) - fqyl))
               + msftx * _col(rdzw) * (fqzl[1:] - fqzl[:nz]))
    ph_low = mass_old * fo - dt * div_low
    fqx_ip1 = ip1(fqx, 2)
    fqy_jp1 = ip1(fqy, 1)
    fqz_kp1, fqz_k = fqz[1:], fqz[:nz]
    pos = lambda a: np.maximum(0.0, a)
    neg = lambda a: np.minimum(0.0, a)
    flux_out = dt * (msftx * msftx * (rdx * (pos(fqx_ip1) - neg(fqx)) + rdy * (pos(fqy_jp1) - neg(fqy)))
                     + msftx * _col(rdzw) * (neg(fqz_kp1) - pos(fqz_k)))
    if opt == 1:
        scale = np.where(flux_out > ph_low, np.maximum(0.0, ph_low / (flux_out + PD_EPS)), 1.0)
        sx = np.roll(scale, 1, 2)
        sy = np.roll(scale, 1, 1)
        fqx_lim = np.where(fqx > 0.0, sx * fqx, np.where(fqx < 0.0, scale * fqx, fqx))
        fqy_lim = np.where(fqy > 0.0, sy * fqy, np.where(fqy < 0.0, scale * fqy, fqy))
        sp = np.concatenate((scale[:1], scale, scale[-1:]), axis=0)
        fqz_lim = np.where(fqz < 0.0, sp[0 : nz + 1] * fqz, np.where(fqz > 0.0, sp[1 : nz + 2] * fqz, fqz))
    elif opt == 2:
        qmax, qmin = fo, fo
        for ax in (2, 1):
            a1, a2 = np.roll(fo, 1, axis=ax), np.roll(fo, -1, axis=ax)
            qmax = np.maximum(qmax, np.maximum(a1, a2))
            qmin = np.minimum(qmin, np.minimum(a1, a2))
        up = np.concatenate((fo[:1], fo[:-1]), axis=0)
        dn = np.concatenate((fo[1:], fo[-1:]), axis=0)
        qmax = np.maximum(qmax, np.maximum(up, dn))
        qmin = np.minimum(qmin, np.minimum(up, dn))
        flux_in = -dt * (msftx * msftx * (rdx * (neg(fqx_ip1) - pos(fqx)) + rdy * (neg(fqy_jp1) - pos(fqy)))
                         + msftx * _col(rdzw) * (pos(fqz_kp1) - neg(fqz_k)))
        ph_hi = qmax * mass_old - ph_low
        ph_lo = ph_low - qmin * mass_old
        s_in = np.where(flux_in > ph_hi, np.maximum(0.0, ph_hi / (flux_in + PD_EPS)), 1.0)
        s_out = np.where(flux_out > ph_lo, np.maximum(0.0, ph_lo / (flux_out + PD_EPS)), 1.0)
        fqx_lim = np.where(fqx > 0.0, np.minimum(s_in, np.roll(s_out, 1, 2)) * fqx,
                           np.minimum(s_out, np.roll(s_in, 1, 2)) * fqx)
        fqy_lim = np.where(fqy > 0.0, np.minimum(s_in, np.roll(s_out, 1, 1)) * fqy,
                           np.minimum(s_out, np.roll(s_in, 1, 1)) * fqy)
        sip = np.concatenate((s_in[:1], s_in, s_in[-1:]), axis=0)
        sop = np.concatenate((s_out[:1], s_out, s_out[-1:]), axis=0)
        fqz_lim = np.where(fqz < 0.0, np.minimum(sip[1 : nz + 2], sop[0 : nz + 1]) * fqz,
                           np.minimum(sop[1 : nz + 2], sip[0 : nz + 1]) * fqz)
    else:
        raise ValueError(f"limiter option {opt} unsupported")
    fx = fqx_lim + fqxl
    fy = fqy_lim + fqyl
    fz = fqz_lim + fqzl
    if spec:
        tend = -msftx * rdx * specified_div(fx, 2)
        tend = tend - msftx * rdy * specified_div(fy, 1)
        return tend - _col(rdzw) * (fz[1:] - fz[:nz])
    tend = -msftx * rdx * (np.roll(fx, -1, 2) - fx)
    tend = tend - msftx * rdy * (np.roll(fy, -1, 1) - fy)
    return tend - _col(rdzw) * (fz[1:] - fz[:nz])


def _vdiv3(f, romq, rdzw, fzm, fzp):
    """flux_advection.py:1362-1407 (u/v vertical flux divergence, -sign(vel) correction)."""
    nz = f.shape[0]
    vflux = np.zeros((nz + 1,) + f.shape[1:])
    q_km2, q_km1, q_k, q_kp1 = f[: nz - 3], f[1 : nz - 2], f[2 : nz - 1], f[3:nz]
    rk = romq[2 : nz - 1]
    flux4 = (7.0 * (q_k + q_km1) - (q_kp1 + q_km2)) / 12.0
    corr = ((q_kp1 - q_km2) - 3.0 * (q_k - q_km1)) / 12.0
    vflux[2 : nz - 1] = rk * (flux4 + np.sign(-rk) * corr)
    vflux[1] = romq[1] * (fzm[1] * f[1] + fzp[1] * f[0])
    vflux[nz - 1] = romq[nz - 1] * (fzm[nz - 1] * f[nz - 1] + fzp[nz - 1] * f[nz - 2])
    return -_col(rdzw) * (vflux[1:] - vflux[:nz])


def _vdiv_w(w, rom, rdn, top_lid):
    """flux_advection.py:1410-1482 (vertical flux divergence of w)."""
    nz = w.shape[0] - 1
    vel = 0.5 * (rom + np.roll(rom, 1, axis=0))
    vflux = np.zeros_like(w)

    def f3(k):
        q_km2, q_km1, q_k, q_kp1 = w[k - 2], w[k - 1], w[k], w[k + 1]
        flux4 = (7.0 * (q_k + q_km1) - (q_kp1 + q_km2)) / 12.0
        corr = ((q_kp1 - q_km2) - 3.0 * (q_k - q_km1)) / 12.0
        return vel[k] * (flux4 + np.sign(-vel[k]) * corr)

    for k in range(3, nz):
        vflux[k] = f3(k)
    vflux[1] = vel[1] * 0.5 * (w[1] + w[0])
    vflux[2] = f3(2)
    vflux[nz - 1] = f3(nz - 1)
    if not top_lid:
        vflux[nz] = vel[nz] * 0.5 * (w[nz] + w[nz - 1])
    tend = np.zeros_like(w)
    tend[1:nz] = -_col(rdn[1:nz]) * (vflux[2 : nz + 1] - vflux[1:nz])
    if not top_lid:
        tend[nz] = tend[nz] + 2.0 * rdn[nz - 1] * vflux[nz]
    return tend


def _advect_u_flux_specified(u, vel, rdx, rdy, m):
    """flux_advection.py:1150-1182: tiers on the full staggered u (upstream
    rule on the normal x faces), faces 1..nx-1 updated."""
    nxs = u.shape[-1]
    msfux = m.msfux[None]
    velx = 0.5 * (vel.ru_full + _shift0(vel.ru_full, 1, 2))
    tend = -msfux * rdx * specified_div(specified_flux_faces(u, velx, 2, upstream=True), 2)
    rv_pad = np.pad(vel.rv_full, ((0, 0), (0, 0), (1, 1)))
    vely = (0.5 * (rv_pad[:, :, 1:] + rv_pad[:, :, :-1]))[:, : u.shape[1], :]
    tend = tend - msfux * rdy * specified_div(specified_flux_faces(u, vely, 1), 1)
    rom_pad = np.pad(vel.rom, ((0, 0), (0, 0), (1, 1)))
    tend = tend + _vdiv3(u, 0.5 * (rom_pad[:, :, 1:] + rom_pad[:, :, :-1]), m.rdnw, m.fnm, m.fnp)
    fi = np.arange(nxs).reshape(1, 1, nxs)
    return np.where((fi >= 1) & (fi <= nxs - 2), tend, 0.0)


def _advect_v_flux_specified(v, vel, rdx, rdy, m):
    """flux_advection.py:1217-1254: the mirror of the u path (upstream rule on
    the normal y faces), rows 1..ny-1 updated."""
    nys = v.shape[-2]
    msfvy, msfvx = m.msfvy[None], m.msfvx[None]
    ru_pad = np.pad(vel.ru_full, ((0, 0), (1, 1), (0, 0)))
    velx = (0.5 * (ru_pad[:, 1:, :] + ru_pad[:, :-1, :]))[:, :, : v.shape[-1]]
    tend = -msfvy * rdx * specified_div(specified_flux_faces(v, velx, 2), 2)
    vely = 0.5 * (vel.rv_full + _shift0(vel.rv_full, 1, 1))
    tend = tend - msfvy * rdy * specified_div(specified_flux_faces(v, vely, 1, upstream=True), 1)
    rom_pad = np.pad(vel.rom, ((0, 0), (1, 1), (0, 0)))
    tend = tend + (msfvy / msfvx) * _vdiv3(v, 0.5 * (rom_pad[:, 1:, :] + rom_pad[:, :-1, :]), m.rdnw, m.fnm, m.fnp)
    ri = np.arange(nys).reshape(1, nys, 1)
    return np.where((ri >= 1) & (ri <= nys - 2), tend, 0.0)


def advect_u_flux(u, vel, rdx, rdy, m):
    """flux_advection.py:1131-1202 (periodic path; specified degrade at :1150-1182)."""
    if getattr(vel, "specified", False):
        return _advect_u_flux_specified(u, vel, rdx, rdy, m)
    nx = vel.ru.shape[-1]
    ny = u.shape[1]
    u_f = u[..., :nx]
    msfux = vel.msfux[None]
    velx = 0.5 * (vel.ru + np.roll(vel.ru, 1, -1))
    fqx = velx * flux5_face(u_f, velx, 2)
    tend = -msfux * rdx * (np.roll(fqx, -1, 2) - fqx)
    if ny > 1:
        vely = 0.5 * (vel.rv + np.roll(vel.rv, 1, -1))
        fqy = vely * flux5_face(u_f, vely, 1)
        tend = tend - msfux * rdy * (np.roll(fqy, -1, 1) - fqy)
    tend = tend + _vdiv3(u_f, 0.5 * (vel.rom + np.roll(vel.rom, 1, -1)), m.rdnw, m.fnm, m.fnp)
    return np.concatenate((tend, tend[:, :, :1]), axis=2)


def advect_v_flux(v, vel, rdx, rdy, m):
    """flux_advection.py:1205-1274 (periodic path; specified degrade at :1217-1254)."""
    if getattr(vel, "specified", False):
        return _advect_v_flux_specified(v, vel, rdx, rdy, m)
    ny = vel.rv.shape[-2]
    v_f = v[:, :ny, :]
    msfvy = vel.msfvy[None]
    msfvx = vel.msfvx[None]
    ru_c = vel.ru[:, :ny, :]
    velx = 0.5 * (ru_c + np.roll(ru_c, 1, -2))
    fqx = velx * flux5_face(v_f, velx, 2)
    tend = -msfvy * rdx * (np.roll(fqx, -1, 2) - fqx)
    vely = 0.5 * (vel.rv + np.roll(vel.rv, 1, -2))
    fqy = vely * flux5_face(v_f, vely, 1)
    tend = tend - msfvy * rdy * (np.roll(fqy, -1, 1) - fqy)
    tend = tend + (msfvy / msfvx) * _vdiv3(v_f, 0.5 * (vel.rom + np.roll(vel.rom, 1, -2)), m.rdnw, m.fnm, m.fnp)
    return np.concatenate((tend, tend[:, :1, :]), axis=1)


def _mass_to_full(f, fzm, fzp):
    """flux_advection.py:1332-1352."""
    nz = f.shape[0]
    out = np.zeros((nz + 1,) + f.shape[1:])
    out[1:nz] = _col(fzm[1:nz]) * f[1:nz] + _col(fzp[1:nz]) * f[: nz - 1]
    out[0] = f[0]
    out[nz] = f[nz - 1]
    return out


def advect_w_flux(w, vel, rdx, rdy, m, top_lid):
    """flux_advection.py:1277-1329 (periodic path; specified degrade at :1305-1318)."""
    msftx = vel.msftx[None]
    ru_w = _mass_to_full(vel.ru, m.fnm, m.fnp)
    rv_w = _mass_to_full(vel.rv, m.fnm, m.fnp)
    if getattr(vel, "specified", False):  # :1305-1318
        tend = -msftx * rdx * specified_div(specified_flux_faces(w, ru_w, 2), 2)
        tend = tend - msftx * rdy * specified_div(specified_flux_faces(w, rv_w, 1), 1)
        return tend + _vdiv_w(w, vel.rom, m.rdn, top_lid)
    fqx = ru_w * flux5_face(w, ru_w, 2)
    tend = -msftx * rdx * (np.roll(fqx, -1, 2) - fqx)
    if w.shape[1] > 1:
        fqy = rv_w * flux5_face(w, rv_w, 1)
        tend = tend - msftx * rdy * (np.roll(fqy, -1, 1) - fqy)
    return tend + _vdiv_w(w, vel.rom, m.rdn, top_lid)


# ----------------------------------------------------------------------------
# large-step PGF / Coriolis: dynamics/core/rk_addtend_dry.py
# ----------------------------------------------------------------------------

def _log_alpha(dph, mass_col, m):
    p_top = float(m.p_top)
    pfu = _col(m.c3f[1:]) * mass_col + _col(m.c4f[1:]) + p_top
    pfd = _col(m.c3f[:-1]) * mass_col + _col(m.c4f[:-1]) + p_top
    phm = _col(m.c3h) * mass_col + _col(m.c4h) + p_top
    return dph / phm / np.log(pfd / pfu)


def absolute_diagnostics(s, m, hyps):
    """rk_addtend_dry.py:127-230 (base_state None)."""
    mub = s.mu_total - s.mu_perturbation
    alt = inv_density(s.theta, s.p_total)
    p_pert = s.p_perturbation
    phb = s.ph_total - s.ph_perturbation
    mass_base = _col(m.c1h) * mub[None] + _col(m.c2h)
    safe_base = np.where(np.abs(mass_base) > 1.0e-12, mass_base, 1.0e-12)
    alb = -_col(m.rdnw) * (phb[1:] - phb[:-1]) / safe_base
    if hyps == 2:
        dph_tot = (phb[1:] + s.ph_perturbation[1:]) - (phb[:-1] + s.ph_perturbation[:-1])
        al = _log_alpha(dph_tot, s.mu_total[None], m) - _log_alpha(phb[1:] - phb[:-1], mub[None], m)
    else:
        muts = s.mu_total + s.mu_perturbation
        mass_t = _col(m.c1h) * muts[None] + _col(m.c2h)
        safe_t = np.where(np.abs(mass_t) > 1.0e-12, mass_t, 1.0e-12)
        mu_term = _col(m.c1h) * s.mu_perturbation[None]
        al = -(alb * mu_term + _col(m.rdnw) * (s.ph_perturbation[1:] - s.ph_perturbation[:-1])) / safe_t
    pht = phb + s.ph_perturbation
    php = 0.5 * (pht[:-1] + pht[1:])
    return s.ph_perturbation, p_pert, al, alt, php


def _cfn(m):
    dn_top = m.dn[-1]
    dn_safe = dn_top if abs(dn_top) > 1.0e-30 else 1.0
    return (0.5 * m.dnw[-1] + m.dn[-1]) / dn_safe, -0.5 * m.dnw[-1] / dn_safe


def large_step_horizontal_pgf(s, m, rdx, rdy, top_lid, hyps):
    """rk_addtend_dry.py:233-362."""
    ph, p_abs, al, alt, php = absolute_diagnostics(s, m, hyps)
    pb = s.p_total - s.p_perturbation
    mub = s.mu_total - s.mu_perturbation
    cqu, cqv = moisture_coupling_factors(s)
    return pgf_from_fields(ph, p_abs, pb, al, alt, php, mub + s.mu_perturbation, s.mu_perturbation, cqu, cqv, m,
                           rdx, rdy, top_lid)


def pgf_dpn(ps, m, top_lid):
    """Face values of a pair sum of pressures for the large-step PGF
    (rk_addtend_dry.py:289-316): half the cf1/cf2/cf3 extrapolation at the
    surface, half the fnm/fnp interpolation inside, the cfn/cfn1 one at a
    rigid lid's top (zero otherwise)."""
    cfn, cfn1 = _cfn(m)
    nz = ps.shape[0]
    dpn = np.zeros((nz + 1,) + ps.shape[1:])
    dpn[0] = 0.5 * (m.cf1 * ps[0] + m.cf2 * ps[1] + m.cf3 * ps[2])
    dpn[1:nz] = 0.5 * (_col(m.fnm[1:]) * ps[1:] + _col(m.fnp[1:]) * ps[:-1])
    if top_lid:
        dpn[nz] = 0.5 * (cfn * ps[-1] + cfn1 * ps[-2])
    return dpn


def pgf_from_fields(ph, p_abs, pb, al, alt, php, mu_total, mu_pert, cqu, cqv, m, rdx, rdy, top_lid,
                    non_hydrostatic=True):
    """The large-step horizontal pressure gradient from its fields
    (rk_addtend_dry.py:233-362; the same terms as acoustic_wrf.py's
    horizontal_pressure_gradient): per u face 0.5 rdx mass_u msf_u times the
    geopotential difference summed over the two adjacent w levels, plus
    (alt_l + alt_r)(p_r - p_l) and (al_l + al_r)(pb_r - pb_l), then (when
    ``non_hydrostatic``) rdx msf_u (php_r - php_l)(rdnw (dpn(k+1) - dpn(k)) -
    0.5 c1 (mu'_l + mu'_r)); returns (-cqu dpx, -cqv dpy)."""
    c1h, c2h, rdnw = _col(m.c1h), _col(m.c2h), _col(m.rdnw)
    msf_u = (m.msfux / m.msfuy)[None]
    msf_v = (m.msfvy / m.msfvx)[None]
    dpn_faces = lambda ps: pgf_dpn(ps, m, top_lid)
    ph_l, ph_r = xpair(ph)
    p_l, p_r = xpair(p_abs)
    pb_l, pb_r = xpair(pb)
    al_l, al_r = xpair(al)
    alt_l, alt_r = xpair(alt)
    a, b = xpair(mu_total)
    muu = 0.5 * (a + b)
    mass_u = c1h * muu[None] + c2h
    dpx = msf_u * 0.5 * rdx * mass_u * (((ph_r[1:] - ph_l[1:]) + (ph_r[:-1] - ph_l[:-1]))
                                        + (alt_l + alt_r) * (p_r - p_l) + (al_l + al_r) * (pb_r - pb_l))
    if non_hydrostatic:
        php_l, php_r = xpair(php)
        dpn = dpn_faces(p_l + p_r)
        mu_l, mu_r = xpair(mu_pert)
        bracket = rdnw * (dpn[1:] - dpn[:-1]) - 0.5 * (c1h * (mu_l + mu_r)[None])
        dpx = dpx + msf_u * rdx * (php_r - php_l) * bracket

    ph_s, ph_n = ypair(ph)
    p_s, p_n = ypair(p_abs)
    pb_s, pb_n = ypair(pb)
    al_s, al_n = ypair(al)
    alt_s, alt_n = ypair(alt)
    a, b = ypair(mu_total)
    muv = 0.5 * (a + b)
    mass_v = c1h * muv[None] + c2h
    dpy = msf_v * 0.5 * rdy * mass_v * (((ph_n[1:] - ph_s[1:]) + (ph_n[:-1] - ph_s[:-1]))
                                        + (alt_s + alt_n) * (p_n - p_s) + (al_s + al_n) * (pb_n - pb_s))
    if non_hydrostatic:
        php_s, php_n = ypair(php)
        dpn = dpn_faces(p_s + p_n)
        mu_s, mu_n = ypair(mu_pert)
        bracket = rdnw * (dpn[1:] - dpn[:-1]) - 0.5 * (c1h * (mu_s + mu_n)[None])
        dpy = dpy + msf_v * rdy * (php_n - php_s) * bracket
    return -cqu * dpx, -cqv * dpy


def large_step_coriolis(s, m, specified):
    """rk_addtend_dry.py:364-484."""
    c1h, c2h, c1f, c2f = _col(m.c1h), _col(m.c2h), _col(m.c1f), _col(m.c2f)
    a, b = xpair(s.mu_total)
    muu = 0.5 * (a + b)
    a, b = ypair(s.mu_total)
    muv = 0.5 * (a + b)
    ru = s.u * (c1h * muu[None] + c2h) / m.msfuy[None]
    rv = s.v * (c1h * muv[None] + c2h) / m.msfvx[None]
    rw = s.w * (c1f * s.mu_total[None] + c2f) / m.msfty[None]

    def xavg(f):
        a, b = xpair(f)
        return 0.5 * (a + b)

    def yavg(f):
        a, b = ypair(f)
        return 0.5 * (a + b)

    f_u, e_u, cosa_u = xavg(m.f), xavg(m.e), xavg(m.cosa)
    f_v, e_v, sina_v = yavg(m.f), yavg(m.e), yavg(m.sina)
    msf_u = (m.msfux / m.msfuy)[None]
    msf_v = (m.msfvy / m.msfvx)[None]
    rv_im1, rv_i = xpair(rv)
    rv_quad = 0.25 * (rv_im1[:, :-1, :] + rv_i[:, :-1, :] + rv_im1[:, 1:, :] + rv_i[:, 1:, :])
    ru_cor = msf_u * f_u[None] * rv_quad
    rw_im1, rw_i = xpair(rw)
    rw_u = 0.25 * (rw_im1[:-1] + rw_im1[1:] + rw_i[:-1] + rw_i[1:])
    ru_cor = ru_cor - e_u[None] * cosa_u[None] * rw_u
    if specified:
        ru_cor[:, :, 0] *= 0.0
        ru_cor[:, :, -1] *= 0.0
    ru_jm1, ru_j = ypair(ru)
    ru_quad = 0.25 * (ru_jm1[:, :, :-1] + ru_jm1[:, :, 1:] + ru_j[:, :, :-1] + ru_j[:, :, 1:])
    rv_cor = -msf_v * f_v[None] * ru_quad
    rw_jm1, rw_j = ypair(rw)
    rw_v = 0.25 * (rw_jm1[:-1] + rw_jm1[1:] + rw_j[:-1] + rw_j[1:])
    rv_cor = rv_cor + msf_v * e_v[None] * sina_v[None] * rw_v
    if specified:
        rv_cor[:, 0, :] *= 0.0
        rv_cor[:, -1, :] *= 0.0
    return ru_cor, rv_cor


# ----------------------------------------------------------------------------
# large-step tendency assembly: runtime/operational_mode.py:2722-3093, 3162-3316
# ----------------------------------------------------------------------------

def rk_addtend_dry(t, physics, rk_step, m, mut):
    """core/rk_addtend_dry.py:490-546: the RK1-fixed physics tendencies merged
    into one stage's tendencies (u, v, w coupled by their map factors, theta
    with the diabatic heating coupled by the full column mass ``mut``; the
    rk_step 1 boundary saves added first).  ``physics`` has the attributes of
    DryPhysicsTendencies (None = zero); ph has no consumer on this path."""
    z = lambda ref, c: np.zeros_like(ref) if c is None else c
    ru, rv, rw = z(t.u, physics.ru_tendf), z(t.v, physics.rv_tendf), z(t.w, physics.rw_tendf)
    tt, mt = z(t.theta, physics.t_tendf), z(t.mu, physics.mu_tendf)
    if rk_step == 1:
        ru = ru + z(t.u, physics.u_save) * m.msfuy[None]
        rv = rv + z(t.v, physics.v_save) * m.msfvx[None]
        rw = rw + z(t.w, physics.w_save) * m.msfty[None]
        tt = tt + z(t.theta, physics.t_save)
    mass_h = _col(m.c1h) * mut[None] + _col(m.c2h)
    h = z(t.theta, physics.h_diabatic)
    return SimpleNamespace(u=t.u + ru / m.msfuy[None], v=t.v + rv * (1.0 / m.msfvx)[None],
                           w=t.w + rw / m.msfty[None],
                           theta=t.theta + tt / m.msfty[None] + mass_h * h / m.msfty[None], mu=t.mu + mt)


def dflux6(f, axis):
    """``_dflux6`` (dynamics/explicit_diffusion.py:160-180): the 6th-order
    diffusive fluxes at the left (p0) and right (p1) faces of every cell and
    the matching first differences, neighbours wrapped along ``axis``."""
    r = lambda n: np.roll(f, n, axis=axis)
    fm3, fm2, fm1, fp1, fp2, fp3 = r(3), r(2), r(1), r(-1), r(-2), r(-3)
    p0 = 10.0 * (f - fm1) - 5.0 * (fp1 - fm2) + (fp2 - fm3)
    p1 = 10.0 * (fp1 - f) - 5.0 * (fp2 - fm1) + (fp3 - fm2)
    return p0, p1, f - fm1, fp1 - f


def sixth_axis(f, axis, coef):
    """``_sixth_axis`` (explicit_diffusion.py:183-197) with the monotonic
    limiter on (the stage passes the default): fluxes that point up-gradient
    are zeroed."""
    p0, p1, g0, g1 = dflux6(f, axis)
    p0 = np.where(p0 * g0 <= 0.0, 0.0, p0)
    p1 = np.where(p1 * g1 <= 0.0, 0.0, p1)
    return coef * (p1 - p0)


def sixth_order_diffusion_tendency(f, dt, factor):
    """``sixth_order_diffusion_tendency`` (explicit_diffusion.py:200-226): the
    uncoupled filter tendency along x, plus along y when the field has more
    than one row; coefficient factor * 0.015625 / (2 dt)."""
    coef = float(factor) * 0.015625 / (2.0 * float(dt))
    t = sixth_axis(f, 2, coef)
    if f.shape[1] > 1:
        t = t + sixth_axis(f, 1, coef)
    return t


PRANDTL = 1.0 / 3.0  # explicit_diffusion.py:956


def horizontal_deformation_2d(u, v, dx, dy):
    """``horizontal_deformation_2d`` (explicit_diffusion.py:960-1113) as the
    stage calls it (operational_mode.py:2950: no metric arguments, so the map
    factors are one and the zx / zy slope terms multiply zero): D11 = 2 du/dx
    and D22 = 2 dv/dy on mass cells, D12 = du/dy + dv/dx on the cell's SW
    corner; u and v without their wrap faces, neighbours rolled."""
    nx = u.shape[2] - 1
    ny = v.shape[1] - 1
    um = u[:, :, :nx]
    vm = v[:, :ny, :]
    d11 = 2.0 * ((np.roll(um, -1, axis=2) - um) / dx)
    d22 = 2.0 * ((np.roll(vm, -1, axis=1) - vm) / dy)
    dudy = (um - np.roll(um, 1, axis=1)) / dy
    dvdx = (vm - np.roll(vm, 1, axis=2)) / dx
    return d11, d22, dudy + dvdx


def smag2d_horizontal_km(d11, d22, d12, dx, dy, c_s):
    """``smag2d_horizontal_km`` (explicit_diffusion.py:1116-1212), unit map
    factors, no slope reduction: the four-corner D12 average, def2, the
    mixing length sqrt(dx dy), xkmh = c_s^2 l^2 sqrt(def2) capped at 10 l,
    xkhh = xkmh / prandtl."""
    nw = np.roll(d12, -1, axis=1)
    se = np.roll(d12, -1, axis=2)
    ne = np.roll(np.roll(d12, -1, axis=1), -1, axis=2)
    tmp = 0.25 * (d12 + nw + se + ne)
    def2 = 0.25 * (d11 - d22) * (d11 - d22) + tmp * tmp
    mlen_h = np.sqrt((dx / 1.0) * (dy / 1.0))
    xkmh = c_s * c_s * mlen_h * mlen_h * np.sqrt(def2)
    xkmh = np.minimum(xkmh, 10.0 * mlen_h)
    return xkmh, xkmh / PRANDTL


def hdiff_coord(field, k, mass, dx, dy):
    """``_hdiff_coord_scalar`` (explicit_diffusion.py:1233-1284): the
    mass-coupled variable-K flux divergence along coordinate surfaces, face K
    and face mass the averages of the two cells, neighbours rolled; the y part
    only for fields with more than one row."""
    rdx, rdy = 1.0 / dx, 1.0 / dy
    r = lambda a, n, ax: np.roll(a, n, axis=ax)
    mkrdxp = 0.5 * (r(k, -1, 2) + k) * (0.5 * (r(mass, -1, 2) + mass)) * rdx
    mkrdxm = 0.5 * (k + r(k, 1, 2)) * (0.5 * (mass + r(mass, 1, 2))) * rdx
    tend = rdx * (mkrdxp * (r(field, -1, 2) - field) - mkrdxm * (field - r(field, 1, 2)))
    if field.shape[1] > 1:
        mkrdyp = 0.5 * (r(k, -1, 1) + k) * (0.5 * (r(mass, -1, 1) + mass)) * rdy
        mkrdym = 0.5 * (k + r(k, 1, 1)) * (0.5 * (mass + r(mass, 1, 1))) * rdy
        tend = tend + rdy * (mkrdyp * (r(field, -1, 1) - field) - mkrdym * (field - r(field, 1, 1)))
    return tend


def k_to_w_levels(k):
    """``_xkmhd_to_w_levels`` (explicit_diffusion.py:1215-1230)."""
    nz = k.shape[0]
    out = np.zeros((nz + 1,) + k.shape[1:])
    out[1:nz] = 0.5 * (k[1:nz] + k[0:nz - 1])
    out[0] = k[0]
    out[nz] = k[nz - 1]
    return out


def smagorinsky_2d_tendencies(s, mass_u, mass_v, mass_h, mass_f, dx, dy, c_s):
    """The diff_opt=1 / km_opt=4 block of the stage (operational_mode.py:
    2946-2960): coupled u, v, w, theta tendencies (theta as the perturbation
    from 300 K, with xkhh; momentum with xkmh on each field's own stagger,
    wrap faces repeated)."""
    d11, d22, d12 = horizontal_deformation_2d(s.u, s.v, dx, dy)
    xkmh, xkhh = smag2d_horizontal_km(d11, d22, d12, dx, dy, c_s)
    nz, ny, nx = s.theta.shape
    th = hdiff_coord(s.theta - T0, xkhh, mass_h, dx, dy)
    du = hdiff_coord(s.u[:, :, :nx], xkmh, mass_u[:, :, :nx], dx, dy)
    dv = hdiff_coord(s.v[:, :ny, :], xkmh, mass_v[:, :ny, :], dx, dy)
    dw = hdiff_coord(s.w, k_to_w_levels(xkmh), mass_f, dx, dy)
    du = np.concatenate((du, du[:, :, :1]), axis=2)
    dv = np.concatenate((dv, dv[:, :1, :]), axis=1)
    return du, dv, dw, th


def const_k_diffusion(field, mass, nu, dx, dy, dz):
    """``conservative_constant_k_diffusion_tendency`` (explicit_diffusion.py:
    282-331): d/dx_j(mass K d field/dx_j), periodic rolls over the field's
    own extent horizontally, zero flux through the bottom and top faces."""
    r = lambda a, n, ax: np.roll(a, n, axis=ax)
    tend = np.zeros_like(field)
    mass_xf = 0.5 * (mass + r(mass, -1, 2))
    fx = mass_xf * nu * (r(field, -1, 2) - field) / dx
    tend = tend + (fx - r(fx, 1, 2)) / dx
    if field.shape[1] > 1:
        mass_yf = 0.5 * (mass + r(mass, -1, 1))
        fy = mass_yf * nu * (r(field, -1, 1) - field) / dy
        tend = tend + (fy - r(fy, 1, 1)) / dy
    nz = field.shape[0]
    if nz > 2:
        mass_zf = 0.5 * (mass[:-1] + mass[1:])
        flux = np.zeros((nz + 1,) + field.shape[1:])
        flux[1:nz] = mass_zf * nu * (field[1:] - field[:-1]) / dz
        tend = tend + (flux[1:] - flux[:nz]) / dz
    return tend


def const_k_dz(ph_total):
    """The stage's mean physical layer depth for the constant-K vertical term
    (operational_mode.py:2757-2758): max(mean(diff(ph)/g), 1)."""
    return max(float(np.mean((ph_total[1:] - ph_total[:-1]) / G)), 1.0)


def augment_large_step_tendencies(s, origin, vel, nl: Namelist, rk_step, bdy_relax=None, physics=None):
    """operational_mode.py:2722-3093 (flux advection on; the 6th-order filter,
    constant-K and 2-D Smagorinsky diffusion when selected), with
    the physics merge (:3062-3075) when ``physics`` is given."""
    m = nl.metrics
    rdx, rdy = 1.0 / nl.dx, 1.0 / nl.dy
    c1h, c2h, c1f, c2f = _col(m.c1h), _col(m.c2h), _col(m.c1f), _col(m.c2f)
    bt = nl.base_tend or {}
    muu = u_face_average_2d(s.mu_total)
    muv = v_face_average_2d(s.mu_total)
    mass_u = c1h * muu[None] + c2h
    mass_v = c1h * muv[None] + c2h
    mass_h = c1h * s.mu_total[None] + c2h
    mass_f = c1f * s.mu_total[None] + c2f
    nz, ny, nx = s.theta.shape
    bu = bt.get("u", np.zeros((nz, ny, nx + 1)))
    bv = bt.get("v", np.zeros((nz, ny + 1, nx)))
    bw = bt.get("w", np.zeros((nz + 1, ny, nx)))
    bth = bt.get("theta", np.zeros((nz, ny, nx)))
    bmu = bt.get("mu", np.zeros((ny, nx)))
    u_t = bu * mass_u + advect_u_flux(s.u, vel, rdx, rdy, m)
    v_t = bv * mass_v + advect_v_flux(s.v, vel, rdx, rdy, m)
    w_t = bw * mass_f + advect_w_flux(s.w, vel, rdx, rdy, m, nl.top_lid)
    use_lim = nl.scalar_adv_opt in (1, 2) and rk_step == 3
    if use_lim:
        adv = advect_scalar_flux_limited(s.theta - T0, origin.theta - T0, vel, nl.scalar_adv_opt,
                                         s.mu_total, origin.mu_total, m, rdx, rdy, nl.dt_s)
    else:
        adv = advect_scalar_flux(s.theta - T0, vel, rdx, rdy, m.rdnw, m.fnm, m.fnp)
    th_t = bth * mass_h + adv
    if nl.diff_6th_opt != 0:  # operational_mode.py:2870-2876
        f6 = nl.diff_6th_factor
        u_t = u_t + mass_u * sixth_order_diffusion_tendency(s.u, nl.dt_s, f6)
        v_t = v_t + mass_v * sixth_order_diffusion_tendency(s.v, nl.dt_s, f6)
        w_t = w_t + mass_f * sixth_order_diffusion_tendency(s.w, nl.dt_s, f6)
        th_t = th_t + mass_h * sixth_order_diffusion_tendency(s.theta, nl.dt_s, f6)
    if nl.const_nu_m2_s > 0.0:  # operational_mode.py:2878-2929 (scalar flux-divergence form)
        nu, dz = float(nl.const_nu_m2_s), const_k_dz(s.ph_total)
        th_t = th_t + const_k_diffusion(s.theta, mass_h, nu, nl.dx, nl.dy, dz)
        u_t = u_t + const_k_diffusion(s.u, mass_u, nu, nl.dx, nl.dy, dz)
        v_t = v_t + const_k_diffusion(s.v, mass_v, nu, nl.dx, nl.dy, dz)
        w_t = w_t + const_k_diffusion(s.w, mass_f, nu, nl.dx, nl.dy, dz)
    if nl.diff_opt == 1 and nl.km_opt == 4:  # operational_mode.py:2946-2960
        du, dv, dw, dth = smagorinsky_2d_tendencies(s, mass_u, mass_v, mass_h, mass_f, nl.dx, nl.dy, nl.c_s)
        th_t = th_t + dth
        u_t = u_t + du
        v_t = v_t + dv
        w_t = w_t + dw
    ru_pgf, rv_pgf = large_step_horizontal_pgf(s, m, rdx, rdy, nl.top_lid, nl.hypsometric_opt)
    u_t = u_t + ru_pgf
    v_t = v_t + rv_pgf
    ru_cor, rv_cor = large_step_coriolis(s, m, bool(nl.run_boundary))
    u_t = u_t + ru_cor
    v_t = v_t + rv_cor
    if physics is not None:
        mg = rk_addtend_dry(SimpleNamespace(u=u_t, v=v_t, w=w_t, theta=th_t, mu=bmu), physics, rk_step, m,
                            s.mu_total)
        u_t, v_t, w_t, th_t, bmu = mg.u, mg.v, mg.w, mg.theta, mg.mu
    if bdy_relax is not None:  # operational_mode.py:3085-3092 (mu at the first stage only)
        return SimpleNamespace(u=u_t + bdy_relax.ru, v=v_t + bdy_relax.rv, w=w_t, theta=th_t + bdy_relax.t,
                               mu=(bmu + bdy_relax.mu) if rk_step == 1 else bmu.copy())
    return SimpleNamespace(u=u_t, v=v_t, w=w_t, theta=th_t, mu=bmu.copy())


def moisture_coupled_tendencies(s, origin, vel, nl: Namelist, rk_step):
    """operational_mode.py:3162-3237 -> flux_advection.py:1002-1100."""
    m = nl.metrics
    rdx, rdy = 1.0 / nl.dx, 1.0 / nl.dy
    use_lim = nl.moist_adv_opt in (1, 2) and rk_step == 3
    out = []
    for name in MOIST_SPECIES:
        q = getattr(s, name)
        if use_lim:
            out.append(advect_scalar_flux_limited(q, getattr(origin, name), vel, nl.moist_adv_opt,
                                                  s.mu_total, origin.mu_total, m, rdx, rdy, nl.dt_s))
        else:
            out.append(advect_scalar_flux(q, vel, rdx, rdy, m.rdnw, m.fnm, m.fnp))
    return out


# ----------------------------------------------------------------------------
# small step prep / calc_p_rho / coefficients
# ----------------------------------------------------------------------------

def small_step_prep(s, ref, rk_step, m, ww):
    """core/small_step_prep.py:216-394 (base_state None)."""
    c1h, c2h, c1f, c2f = _col(m.c1h), _col(m.c2h), _col(m.c1f), _col(m.c2f)
    theta_ref = ref.theta - T0
    theta_cur = s.theta - T0
    mub = s.mu_total - s.mu_perturbation
    mu_cur = s.mu_perturbation
    mu_ref = ref.mu_perturbation
    mu_work = np.zeros_like(mu_cur) if rk_step == 1 else mu_ref - mu_cur
    mut = mub + mu_cur
    muts = mut + mu_work
    muu, muv = u_face_average_2d(mut), v_face_average_2d(mut)
    muus, muvs = u_face_average_2d(muts), v_face_average_2d(muts)
    mass_u_ref, mass_u_cur = c1h * muus[None] + c2h, c1h * muu[None] + c2h
    mass_v_ref, mass_v_cur = c1h * muvs[None] + c2h, c1h * muv[None] + c2h
    mass_h_ref, mass_h_cur = c1h * muts[None] + c2h, c1h * mut[None] + c2h
    mass_f_ref, mass_f_cur = c1f * muts[None] + c2f, c1f * mut[None] + c2f
    p = SimpleNamespace()
    p.rk_step = rk_step
    p.u_work = (mass_u_ref * ref.u - mass_u_cur * s.u) / m.msfuy[None]
    p.v_work = (mass_v_ref * ref.v - mass_v_cur * s.v) / m.msfvx[None]
    p.theta_work = mass_h_ref * theta_ref - mass_h_cur * theta_cur
    p.w_work = (mass_f_ref * ref.w - mass_f_cur * s.w) / m.msfty[None]
    p.ph_work = ref.ph_perturbation - s.ph_perturbation
    alt = inv_density(s.theta, s.p_total)
    p.p_pert = s.p_perturbation
    p.pb = s.p_total - s.p_perturbation
    p.alt = np.maximum(alt, MIN_ACOUSTIC_ALT)
    p.c2a = CPOVCV * (p.pb + p.p_pert) / p.alt
    p.cqu, p.cqv = moisture_coupling_factors(s)
    p.phb = s.ph_total - s.ph_perturbation
    ph = s.ph_perturbation
    p.php = 0.5 * (p.phb[:-1] + p.phb[1:] + ph[:-1] + ph[1:])
    p.ww_save = ww.copy()
    p.theta_1 = theta_ref
    p.ph_1 = ref.ph_perturbation
    p.u_save, p.v_save, p.w_save = s.u, s.v, s.w
    p.t_save = theta_cur
    p.ph_save = s.ph_perturbation
    p.mu_save = mu_cur
    p.mub, p.mut, p.muts, p.mu_work = mub, mut, muts, mu_work
    p.muu, p.muv, p.muus, p.muvs = muu, muv, muus, muvs
    return p


def calc_al_p(mu_work, muts, ph_work, theta_work, theta_1, c2a, alt, m):
    """core/calc_p_rho.py:52-101."""
    mass_h = _col(m.c1h) * muts[None] + _col(m.c2h)
    safe = np.where(np.abs(mass_h) > 1.0e-12, mass_h, 1.0e-12)
    mu_term = _col(m.c1h) * mu_work[None]
    al = -(alt * mu_term + _col(m.rdnw) * (ph_work[1:] - ph_work[:-1])) / safe
    ttr = T0 + theta_1
    sttr = np.where(np.abs(ttr) > 1.0e-6, ttr, 1.0e-6)
    pp = c2a * (alt * (theta_work - mu_term * theta_1) / (safe * sttr) - al)
    return al, pp


def calc_coef_w(mut, m, dts, epssm, top_lid, cqw, c2a):
    """dynamics/acoustic_wrf.py:783-852."""
    nz = m.c1h.shape[0]
    ny, nx = mut.shape
    mass_h = _col(m.c1h) * mut[None] + _col(m.c2h)
    mass_f = _col(m.c1f) * mut[None] + _col(m.c2f)
    rdn, rdnw = m.rdn, m.rdnw
    cof = (0.5 * dts * G * (1.0 + epssm)) ** 2
    lid = 0.0 if top_lid else 1.0
    a = np.zeros((nz + 1, ny, nx))
    alpha = np.ones((nz + 1, ny, nx))
    gamma = np.zeros((nz + 1, ny, nx))
    a[nz] = -2.0 * cof * rdnw[nz - 1] ** 2 * c2a[nz - 1] * lid / (mass_h[nz - 1] * mass_f[nz - 1])
    for kk in range(2, nz):
        k = kk - 1
        a[kk] = -cqw[kk] * cof * rdn[kk] * rdnw[kk - 1] * c2a[kk - 1] / (mass_h[k] * mass_f[k])
    for k in range(1, nz):
        b = 1.0 + cqw[k] * cof * rdn[k] * (rdnw[k] * c2a[k] / (mass_h[k] * mass_f[k])
                                           + rdnw[k - 1] * c2a[k - 1] / (mass_h[k - 1] * mass_f[k]))
        c = -cqw[k] * cof * rdn[k] * rdnw[k] * c2a[k] / (mass_h[k] * mass_f[k + 1])
        alpha[k] = 1.0 / (b - a[k] * gamma[k - 1])
        gamma[k] = c * alpha[k]
    b_top = 1.0 + 2.0 * cof * rdnw[nz - 1] ** 2 * c2a[nz - 1] / (mass_h[nz - 1] * mass_f[nz])
    alpha[nz] = 1.0 / (b_top - a[nz] * gamma[nz - 1])
    gamma[nz] = 0.0
    return a, alpha, gamma


def pg_buoy_w_moist(p, mu_prime, mub, qtot, m):
    """core/advance_w.py:195-290 (moist form; identical to dry when qtot == 0)."""
    nz = p.shape[0]
    cqw_calc = np.zeros((nz + 1,) + p.shape[1:])
    cqw_calc[1:nz] = 0.5 * (qtot[1:nz] + qtot[: nz - 1])
    minv = (1.0 / m.msfty)[None]
    rw = np.zeros_like(cqw_calc)
    cqw = np.zeros_like(cqw_calc)
    ci = cqw_calc[1:nz]
    cq1 = 1.0 / (1.0 + ci)
    cq2 = ci * cq1
    rw[1:nz] = minv * G * (cq1 * _col(m.rdn[1:nz]) * (p[1:nz] - p[: nz - 1]) - _col(m.c1f[1:nz]) * mu_prime[None]
                           - cq2 * (_col(m.c1f[1:nz]) * mub[None] + _col(m.c2f[1:nz])))
    cqw[1:nz] = cq1
    ct = cqw_calc[nz - 1]
    c1t = 1.0 / (1.0 + ct)
    c2t = ct * c1t
    rw[nz] = minv[0] * G * (c1t * 2.0 * m.rdnw[nz - 1] * (-p[nz - 1]) - m.c1f[nz] * mu_prime - c2t * (m.c1f[nz] * mub + m.c2f[nz]))
    return rw, cqw


def pg_buoy_w_dry(p, mu_prime, m):
    """core/advance_w.py:146-192."""
    nz = p.shape[0]
    minv = (1.0 / m.msfty)[None]
    rw = np.zeros((nz + 1,) + p.shape[1:])
    rw[1:nz] = minv * G * (_col(m.rdn[1:nz]) * (p[1:nz] - p[: nz - 1]) - _col(m.c1f[1:nz]) * mu_prime[None])
    rw[nz] = minv[0] * G * (2.0 * m.rdnw[nz - 1] * (-p[nz - 1]) - m.c1f[nz] * mu_prime)
    cqw = np.zeros_like(rw)
    cqw[1:nz] = 1.0
    return rw, cqw


def _ph_adv_order6(a, flow_y, flow_x):
    """Order<=6 horizontal phi advection sums under specified lateral BCs
    (core/rhs_ph.py:87-173): per mass row j the y sum is 6th order on rows
    3..ny-4, 4th order on rows 2 and ny-3, 2nd order on rows 1 and ny-2, none
    on rows 0 and ny-1; per column i the x sum is 6th order on 3..nx-4, 2nd
    order on 1 and nx-2, none on 0, 2, nx-3 and nx-1.  ``a`` is phi_total on
    the faces' level(s), ``flow_y``/``flow_x`` the mass-weighted v/u face
    flows.  Each branch is added as a masked term (where-sum order)."""
    ny, nx = a.shape[-2], a.shape[-1]
    lead = ((0, 0),) * (a.ndim - 2)
    py = np.pad(a, lead + ((3, 3), (0, 0)))
    d1 = py[..., 4:-2, :] - py[..., 2:-4, :]
    d2 = py[..., 5:-1, :] - py[..., 1:-5, :]
    d3 = py[..., 6:, :] - py[..., :-6, :]
    dn = py[..., 4:-2, :] - py[..., 3:-3, :]
    ds = py[..., 3:-3, :] - py[..., 2:-4, :]
    fn, fs = flow_y[..., 1:, :], flow_y[..., :-1, :]
    jj = np.arange(ny)[:, None]
    adv_y = np.where((jj >= 3) & (jj <= ny - 4), (fn + fs) * ((45.0 * d1 - 9.0 * d2 + d3) / 60.0), 0.0)
    adv_y = adv_y + np.where((jj == 2) | (jj == ny - 3), (fn + fs) * ((8.0 * d1 - d2) / 12.0), 0.0)
    adv_y = adv_y + np.where((jj == 1) | (jj == ny - 2), fn * dn + fs * ds, 0.0)
    px = np.pad(a, lead + ((0, 0), (3, 3)))
    e1 = px[..., 4:-2] - px[..., 2:-4]
    e2 = px[..., 5:-1] - px[..., 1:-5]
    e3 = px[..., 6:] - px[..., :-6]
    de = px[..., 4:-2] - px[..., 3:-3]
    dw = px[..., 3:-3] - px[..., 2:-4]
    fe, fw = flow_x[..., 1:], flow_x[..., :-1]
    ii = np.arange(nx)[None, :]
    adv_x = np.where((ii >= 3) & (ii <= nx - 4), (fe + fw) * ((45.0 * e1 - 9.0 * e2 + e3) / 60.0), 0.0)
    adv_x = adv_x + np.where((ii == 1) | (ii == nx - 2), fe * de + fw * dw, 0.0)
    return adv_y, adv_x


def rhs_ph(u, v, ww, ph, phb, w, mut, muu, muv, m, rdx, rdy, top_lid, order=2, specified=False):
    """core/rhs_ph.py:175-401: the vertical terms, then the horizontal phi
    advection -- order 2 periodic (:347-401), or the order<=6 specified
    branch (:281-345, with the open-top face row) when order >= 4 under
    specified lateral BCs."""
    if order >= 4 and specified:
        return _rhs_ph_order6_specified(u, v, ww, ph, phb, w, mut, muu, muv, m, rdx, rdy, top_lid)
    return rhs_ph_order2(u, v, ww, ph, phb, w, mut, muu, muv, m, rdx, rdy, top_lid)


def _rhs_ph_vertical(ww, ph, phb, w, mut, m, top_lid):
    """term3 (-omega dphi/deta) and gw of core/rhs_ph.py:248-279."""
    nz = ph.shape[0] - 1
    pht = ph + phb
    minv = (1.0 / m.msfty)[None]
    out = np.zeros_like(ph)
    dphi = pht[1:] - pht[:-1]
    wdwn = 0.5 * (ww[1:] + ww[:-1]) * _col(m.rdnw) * dphi
    term3 = _col(m.fnm[1:nz]) * wdwn[1:nz] + _col(m.fnp[1:nz]) * wdwn[: nz - 1]
    out[1:nz] = out[1:nz] + (-term3)
    mass_f = _col(m.c1f) * mut[None] + _col(m.c2f)
    gw = mass_f * G * w * minv
    out[1:nz] = out[1:nz] + gw[1:nz]
    out[nz] = 0.0 if top_lid else gw[nz]
    return out, pht


def _rhs_ph_order6_specified(u, v, ww, ph, phb, w, mut, muu, muv, m, rdx, rdy, top_lid):
    """core/rhs_ph.py:281-345 with :87-173."""
    nz = ph.shape[0] - 1
    out, pht = _rhs_ph_vertical(ww, ph, phb, w, mut, m, top_lid)
    c1f_int = _col(m.c1f[1:nz])
    c2f_int = _col(m.c2f[1:nz])
    flow_y = (c1f_int * muv[None] + c2f_int) * (v[1:nz] + v[: nz - 1]) * m.msfvy[None]
    flow_x = (c1f_int * muu[None] + c2f_int) * (u[1:nz] + u[: nz - 1]) * m.msfux[None]
    adv_y, adv_x = _ph_adv_order6(pht[1:nz], flow_y, flow_x)
    adv = 0.25 * rdy / m.msfty[None] * adv_y + 0.25 * rdx / m.msfty[None] * adv_x
    out[1:nz] = out[1:nz] + (-adv)
    if not top_lid and nz >= 3:
        cfn, cfn1 = _cfn(m)
        v_top = cfn * v[nz - 1] + cfn1 * v[nz - 2]
        u_top = cfn * u[nz - 1] + cfn1 * u[nz - 2]
        fy = (m.c1f[nz] * muv + m.c2f[nz]) * v_top * m.msfvy
        fx = (m.c1f[nz] * muu + m.c2f[nz]) * u_top * m.msfux
        ay, ax = _ph_adv_order6(pht[nz], fy, fx)
        out[nz] = out[nz] + (-(0.5 * rdy / m.msfty) * ay - (0.5 * rdx / m.msfty) * ax)
    return out


def rhs_ph_order2(u, v, ww, ph, phb, w, mut, muu, muv, m, rdx, rdy, top_lid):
    """core/rhs_ph.py:175-401 (advective_order <= 2 periodic path)."""
    nz = ph.shape[0] - 1
    pht = ph + phb
    minv = (1.0 / m.msfty)[None]
    out = np.zeros_like(ph)
    dphi = pht[1:] - pht[:-1]
    wdwn = 0.5 * (ww[1:] + ww[:-1]) * _col(m.rdnw) * dphi
    term3 = _col(m.fnm[1:nz]) * wdwn[1:nz] + _col(m.fnp[1:nz]) * wdwn[: nz - 1]
    out[1:nz] = out[1:nz] + (-term3)
    mass_f = _col(m.c1f) * mut[None] + _col(m.c2f)
    gw = mass_f * G * w * minv
    out[1:nz] = out[1:nz] + gw[1:nz]
    out[nz] = 0.0 if top_lid else gw[nz]
    c1f_int = _col(m.c1f[1:nz])
    c2f_int = _col(m.c2f[1:nz])
    v_pair = v[1:nz] + v[: nz - 1]
    muvf = c1f_int * muv[None] + c2f_int
    pti = pht[1:nz]
    dn_ = np.roll(pti, -1, -2) - pti
    ds_ = pti - np.roll(pti, 1, -2)
    flux_y = muvf[:, 1:, :] * v_pair[:, 1:, :] * dn_ + muvf[:, :-1, :] * v_pair[:, :-1, :] * ds_
    out[1:nz] = out[1:nz] + (-(0.25 * rdy * minv) * flux_y)
    u_pair = u[1:nz] + u[: nz - 1]
    muuf = c1f_int * muu[None] + c2f_int
    de_ = np.roll(pti, -1, -1) - pti
    dw_ = pti - np.roll(pti, 1, -1)
    flux_x = muuf[:, :, 1:] * u_pair[:, :, 1:] * de_ + muuf[:, :, :-1] * u_pair[:, :, :-1] * dw_
    out[1:nz] = out[1:nz] + (-(0.25 * rdx * minv) * flux_x)
    return out


# ----------------------------------------------------------------------------
# lateral boundary in-step pieces: coupling/boundary_apply.py
# ----------------------------------------------------------------------------

def interpolate_boundary_leaf(leaf, lead_seconds, cadence):
    """boundary_apply.py:329-345."""
    mx = leaf.shape[0] - 1
    li = float(lead_seconds) / float(cadence)
    lo = int(np.clip(np.floor(li), 0, mx))
    hi = int(np.clip(lo + 1, 0, mx))
    a = float(np.clip(li - lo, 0.0, 1.0))
    return leaf[lo] * (1.0 - a) + leaf[hi] * a


def _strip(forcing, side, b, z_len, side_len):
    """boundary_apply.py:528-549."""
    sv = forcing[SIDES.index(side)]
    b = min(max(int(b), 0), sv.shape[0] - 1)
    return sv[b, :z_len, :side_len]


# ---- specified-domain boundary cadence (boundary_apply.py:948-1043, 1148-1340) ----
SPEC_PLUS_RELAX = 5  # spec_zone + relax_zone of the default boundary configuration


def full_ring_target(leaf, z_len, y_len, x_len):
    """boundary_apply.py:948-969: the leaf's strips written into the outer
    five rows / columns (W, E, S, N per width index, later writes win)."""
    t = np.zeros((z_len, y_len, x_len))
    for b in range(SPEC_PLUS_RELAX):
        t[:, :, b] = _strip(leaf, "W", b, z_len, y_len)
        t[:, :, x_len - 1 - b] = _strip(leaf, "E", b, z_len, y_len)
        t[:, b, :] = _strip(leaf, "S", b, z_len, x_len)
        t[:, y_len - 1 - b, :] = _strip(leaf, "N", b, z_len, x_len)
    return t


def _wrf_relax_weights(b, dt, spec_zone=1, relax_zone=4):
    """boundary_apply.py:666-688 (spec_exp 0): dt*fcx, dt*gcx."""
    loop = b + 1
    linear = max(0.0, float(spec_zone + relax_zone - loop) / float(relax_zone - 1))
    fcx = 0.1 / float(dt) * linear * 1.0
    gcx = 1.0 / float(dt) / 50.0 * linear * 1.0
    return float(dt) * fcx, float(dt) * gcx


def _shift_clamp(v, shift, axis):
    """boundary_apply.py:577-586."""
    n = v.shape[axis]
    idx = np.concatenate(([0], np.arange(n - 1))) if shift == 1 else np.concatenate((np.arange(1, n), [n - 1]))
    return np.take(v, idx, axis=axis)


def _relax_tendency_row(f, t, side, b, fcx, gcx):
    """boundary_apply.py:972-1006."""
    if side == "W":
        cur, te, ti, b0, be, bi = f[:, :, b], f[:, :, b - 1], f[:, :, b + 1], t[:, :, b], t[:, :, b - 1], t[:, :, b + 1]
    elif side == "E":
        x = f.shape[2] - 1 - b
        cur, te, ti, b0, be, bi = f[:, :, x], f[:, :, x + 1], f[:, :, x - 1], t[:, :, x], t[:, :, x + 1], t[:, :, x - 1]
    elif side == "S":
        cur, te, ti, b0, be, bi = f[:, b, :], f[:, b - 1, :], f[:, b + 1, :], t[:, b, :], t[:, b - 1, :], t[:, b + 1, :]
    else:
        y = f.shape[1] - 1 - b
        cur, te, ti, b0, be, bi = f[:, y, :], f[:, y + 1, :], f[:, y - 1, :], t[:, y, :], t[:, y + 1, :], t[:, y - 1, :]
    fls0 = b0 - cur
    fls1 = _shift_clamp(fls0, +1, 1)
    fls2 = _shift_clamp(fls0, -1, 1)
    lap = fls1 + fls2 + (be - te) + (bi - ti) - 4.0 * fls0
    return float(fcx) * fls0 - float(gcx) * lap


def scatter_relax_tendency(f, t, dt_full, spec_zone=1, relax_zone=4):
    """boundary_apply.py:1009-1043: the relax-zone tendency with WRF's corner trims."""
    z_len, y_len, x_len = f.shape
    tend = np.zeros_like(f)
    for b in range(spec_zone, relax_zone):
        fcx, gcx = _wrf_relax_weights(b, dt_full, spec_zone, relax_zone)
        fcx, gcx = fcx / float(dt_full), gcx / float(dt_full)
        for side in SIDES:
            row = _relax_tendency_row(f, t, side, b, fcx, gcx)
            if side in ("W", "E"):
                col = b if side == "W" else x_len - 1 - b
                tend[:, b + 1:y_len - b - 1, col] = tend[:, b + 1:y_len - b - 1, col] + row[:, b + 1:y_len - b - 1]
            else:
                r = b if side == "S" else y_len - 1 - b
                tend[:, r, b:x_len - b] = tend[:, r, b:x_len - b] + row[:, b:x_len - b]
    return tend


def specified_relax_dry_tendencies(ref, lead_seconds, m, dt_full, cadence):
    """boundary_apply.py:1148-1248: relax_bdy_dry from the step-start state,
    targets at the step-start lead, both sides coupled with the step-start mass."""
    mu = ref.mu_total
    muu = 0.5 * (np.concatenate([mu[:, :1], mu], axis=1) + np.concatenate([mu, mu[:, -1:]], axis=1))
    muv = 0.5 * (np.concatenate([mu[:1, :], mu], axis=0) + np.concatenate([mu, mu[-1:, :]], axis=0))
    nz, ny, nx = ref.theta.shape
    lf = lambda leaf: interpolate_boundary_leaf(leaf, lead_seconds, cadence)
    u_t = full_ring_target(lf(ref.u_bdy), nz, ny, nx + 1)
    v_t = full_ring_target(lf(ref.v_bdy), nz, ny + 1, nx)
    t_t = full_ring_target(lf(ref.theta_bdy), nz, ny, nx)
    ph_t = full_ring_target(lf(ref.ph_bdy), nz + 1, ny, nx)
    mu_t = full_ring_target(lf(ref.mu_bdy), 1, ny, nx)[0]
    c1h, c2h, c1f, c2f = _col(m.c1h), _col(m.c2h), _col(m.c1f), _col(m.c2f)
    mass_u = c1h * muu[None] + c2h
    mass_v = c1h * muv[None] + c2h
    mass_h = c1h * mu[None] + c2h
    mass_f = c1f * mu[None] + c2f
    r = SimpleNamespace()
    r.ru = scatter_relax_tendency(mass_u * ref.u / m.msfuy[None], mass_u * u_t / m.msfuy[None], dt_full)
    r.rv = scatter_relax_tendency(mass_v * ref.v / m.msfvx[None], mass_v * v_t / m.msfvx[None], dt_full)
    r.t = scatter_relax_tendency(mass_h * ref.theta, mass_h * t_t, dt_full) / m.msfty[None]
    r.ph = scatter_relax_tendency(mass_f * ref.ph_perturbation, mass_f * ph_t, dt_full) / m.msfty[None]
    r.mu = scatter_relax_tendency(ref.mu_perturbation[None], mu_t[None], dt_full)[0]
    return r


def nested_relax_tendency(field, target, mut, m, dt_full):
    """boundary_apply.py:1045-1087: the nested child's relax-zone tendency of a
    full-level field (ph' or w) toward its full-ring target, both coupled with
    c1f*mut+c2f, over msfty."""
    mass_f = _col(m.c1f) * mut[None] + _col(m.c2f)
    return scatter_relax_tendency(mass_f * field, mass_f * target, float(dt_full)) / m.msfty[None]


def tangential_targets(u_strip, v_strip, prep, m):
    """boundary_apply.py:1251-1296 (spec_zone 1): ring-0 work targets of the
    tangential winds, u on the S / N rows, v on the W / E columns."""
    c1h, c2h = _col(m.c1h), _col(m.c2h)
    mu_cur, mu_stg = c1h * prep.muu[None] + c2h, c1h * prep.muus[None] + c2h
    mv_cur, mv_stg = c1h * prep.muv[None] + c2h, c1h * prep.muvs[None] + c2h
    u_save, v_save = prep.u_save, prep.v_save
    nz, ny, nxu = u_save.shape
    _, nyv, nx = v_save.shape
    tu = np.zeros_like(u_save)
    for rr, side in ((0, "S"), (ny - 1, "N")):
        st = _strip(u_strip, side, 0, nz, nxu)
        tu[:, rr, :] = (st * mu_stg[:, rr, :] - u_save[:, rr, :] * mu_cur[:, rr, :]) / m.msfuy[rr, :][None, :]
    tv = np.zeros_like(v_save)
    for cc, side in ((0, "W"), (nx - 1, "E")):
        st = _strip(v_strip, side, 0, nz, nyv)
        tv[:, :, cc] = (st * mv_stg[:, :, cc] - v_save[:, :, cc] * mv_cur[:, :, cc]) / m.msfvx[:, cc][None, :]
    return tu, tv


def _pin_ring(field, target):
    """Ring-0 copy (operational acoustic core :902-915, spec_zone 1)."""
    out = field.copy()
    out[..., 0, :] = target[..., 0, :]
    out[..., -1, :] = target[..., -1, :]
    out[..., :, 0] = target[..., :, 0]
    out[..., :, -1] = target[..., :, -1]
    return out


def specified_w_zero_grad(w_work, w_save, mut, muts, m):
    """core/acoustic.py:383-516 (spec_zone 1): the ring-0 work w whose finished
    physical w equals the nearest interior physical w (S / N rows own corners)."""
    c1f, c2f = _col(m.c1f), _col(m.c2f)
    mass_cur = c1f * mut[None] + c2f
    mass_stage = c1f * muts[None] + c2f
    msfty = m.msfty
    phys = (msfty[None] * w_work + w_save * mass_cur) / mass_stage
    nzp, ny, nx = w_work.shape
    out = w_work.copy()
    xi = np.clip(np.arange(nx), 1, nx - 2)
    work = lambda tgt, j, i: (tgt * mass_stage[:, j, i] - w_save[:, j, i] * mass_cur[:, j, i]) / msfty[j, i]
    out[:, 0, :] = work(phys[:, 1, xi], 0, slice(None))
    out[:, ny - 1, :] = work(phys[:, ny - 2, xi], ny - 1, slice(None))
    rows = np.arange(1, ny - 1)
    yi = np.clip(rows, 1, ny - 2)
    out[:, 1:ny - 1, 0] = work(phys[:, yi, 1], slice(1, ny - 1), 0)
    out[:, 1:ny - 1, nx - 1] = work(phys[:, yi, nx - 2], slice(1, ny - 1), nx - 1)
    return out


def normal_bdy_work_target_u(strip, u_save, mass_cur, mass_stage, msfuy, nzone):
    """boundary_apply.py:729-758."""
    z, y, x = u_save.shape
    t = np.zeros_like(u_save)
    for b in range(nzone):
        ws, es = _strip(strip, "W", b, z, y), _strip(strip, "E", b, z, y)
        cw, ce = b, x - 1 - b
        t[:, :, cw] = (ws * mass_stage[:, :, cw] - u_save[:, :, cw] * mass_cur[:, :, cw]) / msfuy[:, cw][None]
        t[:, :, ce] = (es * mass_stage[:, :, ce] - u_save[:, :, ce] * mass_cur[:, :, ce]) / msfuy[:, ce][None]
    return t


def normal_bdy_work_target_v(strip, v_save, mass_cur, mass_stage, msfvx, nzone):
    """boundary_apply.py:761-781."""
    z, y, x = v_save.shape
    t = np.zeros_like(v_save)
    for b in range(nzone):
        ss, ns = _strip(strip, "S", b, z, x), _strip(strip, "N", b, z, x)
        rs, rn = b, y - 1 - b
        t[:, rs, :] = (ss * mass_stage[:, rs, :] - v_save[:, rs, :] * mass_cur[:, rs, :]) / msfvx[rs, :][None]
        t[:, rn, :] = (ns * mass_stage[:, rn, :] - v_save[:, rn, :] * mass_cur[:, rn, :]) / msfvx[rn, :][None]
    return t


def normal_relax_weights(y_len, x_len, sub_ratio, axis, spec_zone=1, relax_zone=4):
    """boundary_apply.py:803-855 (DEFAULT_BOUNDARY_CONFIG spec/relax widths)."""
    w = np.zeros((y_len, x_len))
    for b in range(spec_zone):
        if axis == "u":
            w[:, b] = 1.0
            w[:, x_len - 1 - b] = 1.0
        else:
            w[b, :] = 1.0
            w[y_len - 1 - b, :] = 1.0
    for b in range(spec_zone, relax_zone):
        linear = max(0.0, (spec_zone + relax_zone - (b + 1)) / float(relax_zone - 1)) if relax_zone > 1 else 0.0
        weight = min(1.0, max(0.0, sub_ratio * 0.1 * linear))
        if axis == "u":
            w[b + 1 : y_len - b - 1, b] = weight
            w[b + 1 : y_len - b - 1, x_len - 1 - b] = weight
        else:
            w[b, b : x_len - b] = weight
            w[y_len - 1 - b, b : x_len - b] = weight
    return w[None]


# ----------------------------------------------------------------------------
# acoustic substep: core/acoustic.py, dynamics/mu_t_advance.py, core/advance_w.py
# ----------------------------------------------------------------------------

def _dpn_acoustic(ps, m, top_lid):
    """core/acoustic.py:563-580."""
    nz = ps.shape[0]
    dpn = np.zeros((nz + 1,) + ps.shape[1:])
    dpn[0] = 0.5 * (m.cf1 * ps[0] + m.cf2 * ps[1] + m.cf3 * ps[2])
    dpn[1:nz] = 0.5 * (_col(m.fnm[1:]) * ps[1:] + _col(m.fnp[1:]) * ps[:-1])
    if top_lid:
        dpn[nz] = 0.5 * (m.cf1 * ps[-1] + m.cf2 * ps[-2] + m.cf3 * ps[-3])
    return dpn


def advance_uv(a, m, dts, rdx, rdy, dx, dy, top_lid, bdy=None):
    """core/acoustic.py:626-786 (emdiv = 0.01)."""
    u = a.u + dts * a.u_tend
    v = a.v + dts * a.v_tend
    c1h, c2h, rdnw = _col(m.c1h), _col(m.c2h), _col(m.rdnw)
    ph_l, ph_r = xpair(a.ph)
    p_l, p_r = xpair(a.p)
    pb_l, pb_r = xpair(a.pb)
    al_l, al_r = xpair(a.al)
    alt_l, alt_r = xpair(a.alt)
    mass_x = c1h * a.muu[None] + c2h
    dpx = (m.msfux / m.msfuy)[None] * 0.5 * rdx * mass_x * (((ph_r[1:] - ph_l[1:]) + (ph_r[:-1] - ph_l[:-1]))
                                                             + (alt_l + alt_r) * (p_r - p_l) + (al_l + al_r) * (pb_r - pb_l))
    php_l, php_r = xpair(a.php)
    dpn = _dpn_acoustic(p_l + p_r, m, top_lid)
    mu_work = a.muts - a.mut
    mu_l, mu_r = xpair(mu_work)
    bracket = rdnw * (dpn[1:] - dpn[:-1]) - 0.5 * (c1h * (mu_l + mu_r)[None])
    dpx = dpx + (m.msfux / m.msfuy)[None] * rdx * (php_r - php_l) * bracket
    u = u - dts * a.cqu * dpx
    md_l, md_r = xpair(a.mudf)
    u = u + c1h * (-EMDIV * dx * (md_r - md_l) / m.msfuy)[None]

    ph_s, ph_n = ypair(a.ph)
    p_s, p_n = ypair(a.p)
    pb_s, pb_n = ypair(a.pb)
    al_s, al_n = ypair(a.al)
    alt_s, alt_n = ypair(a.alt)
    mass_y = c1h * a.muv[None] + c2h
    dpy = (m.msfvy / m.msfvx)[None] * 0.5 * rdy * mass_y * (((ph_n[1:] - ph_s[1:]) + (ph_n[:-1] - ph_s[:-1]))
                                                             + (alt_s + alt_n) * (p_n - p_s) + (al_s + al_n) * (pb_n - pb_s))
    php_s, php_n = ypair(a.php)
    dpn = _dpn_acoustic(p_s + p_n, m, top_lid)
    mu_s, mu_n = ypair(mu_work)
    bracket = rdnw * (dpn[1:] - dpn[:-1]) - 0.5 * (c1h * (mu_s + mu_n)[None])
    dpy = dpy + (m.msfvy / m.msfvx)[None] * rdy * (php_n - php_s) * bracket
    v = v - dts * a.cqv * dpy
    md_s, md_n = ypair(a.mudf)
    v = v + c1h * (-EMDIV * dy * (md_n - md_s) * (1.0 / m.msfvx))[None]
    if bdy is not None:
        u = u + bdy.wu * (bdy.u_target - u)
        v = v + bdy.wv * (bdy.v_target - v)
    a.u, a.v = u, v


def advance_mu_t(a, m, dts, rdx, rdy, epssm, specified):
    """dynamics/mu_t_advance.py:131-292 (periodic) and :295-451 (specified)."""
    nz = a.theta_work.shape[0]
    ny, nx = a.mu.shape
    msfvx_inv = 1.0 / m.msfvx
    if specified:
        y0, y1, x0, x1 = 1, ny - 1, 1, nx - 1
    else:
        y0, y1, x0, x1 = 0, ny, 0, nx
    ys, xs = slice(y0, y1), slice(x0, x1)
    ysn, xse = slice(y0 + 1, y1 + 1), slice(x0 + 1, x1 + 1)
    msftx, msfty = m.msftx[ys, xs], m.msfty[ys, xs]
    dvdxi = np.zeros((nz, y1 - y0, x1 - x0))
    for k in range(nz):
        c1, c2 = m.c1h[k], m.c2h[k]
        vn = a.v[k, ysn, xs] + (c1 * a.muv[ysn, xs] + c2) * a.v_1[k, ysn, xs] * msfvx_inv[ysn, xs]
        vs = a.v[k, ys, xs] + (c1 * a.muv[ys, xs] + c2) * a.v_1[k, ys, xs] * msfvx_inv[ys, xs]
        ue = a.u[k, ys, xse] + (c1 * a.muu[ys, xse] + c2) * a.u_1[k, ys, xse] / m.msfuy[ys, xse]
        uw = a.u[k, ys, xs] + (c1 * a.muu[ys, xs] + c2) * a.u_1[k, ys, xs] / m.msfuy[ys, xs]
        dvdxi[k] = msftx * msfty * (rdy * (vn - vs) + rdx * (ue - uw))
    dmdt = np.sum(_col(m.dnw) * dvdxi, axis=0)
    mu_work_old = a.muts[ys, xs] - a.mut[ys, xs]
    mu_save = a.mu[ys, xs] - mu_work_old
    mu_tend = a.mu_tend[ys, xs]
    mu_tendency = dmdt + mu_tend
    if specified:
        mutc = a.mut[ys, xs]
        floor = np.maximum(MIN_MUTS_PA, MIN_MUTS_FRACTION * mutc)
        muts_old = mutc + mu_work_old
        raw = dts * mu_tendency
        allowed = np.maximum(muts_old - floor, 0.0)
        loss = -raw
        finite = np.isfinite(raw) & np.isfinite(muts_old)
        scale = np.where(finite & (loss > allowed), allowed / np.maximum(loss, 1.0), np.where(finite, 1.0, 0.0))
        scale = np.clip(scale, 0.0, 1.0)
        mu_tendency = mu_tendency * scale
        dmdt = dmdt * scale
        dvdxi = dvdxi * scale[None]
        mu_tend = mu_tend * scale
    mu_work_new = mu_work_old + dts * mu_tendency
    a.mu[ys, xs] = mu_save + mu_work_new
    a.mudf[ys, xs] = mu_tendency
    a.muts[ys, xs] = a.mut[ys, xs] + mu_work_new
    a.muave[ys, xs] = 0.5 * ((1.0 + epssm) * mu_work_new + (1.0 - epssm) * mu_work_old)
    rows = [a.ww[0, ys, xs]]
    for kk in range(1, nz):
        k = kk - 1
        inc = m.dnw[kk - 1] * (m.c1h[k] * dmdt + dvdxi[kk - 1] + m.c1h[k] * mu_tend) / msfty
        rows.append(rows[-1] - inc)
    rows.append(a.ww[nz, ys, xs])
    wwa = np.stack(rows, axis=0)
    wwa[:nz] = wwa[:nz] - a.ww_1[:nz, ys, xs]
    a.ww[:, ys, xs] = wwa
    th1 = a.theta_1
    theta_i = a.theta_work[:, ys, xs] + msfty[None] * dts * a.theta_tend[:, ys, xs]
    wdtn = np.zeros((nz + 1, y1 - y0, x1 - x0))
    for k in range(1, nz):
        wdtn[k] = wwa[k] * (m.fnm[k] * th1[k, ys, xs] + m.fnp[k] * th1[k - 1, ys, xs])
    for k in range(nz):
        th = th1[k]
        if specified:
            th_e, th_w = th[ys, x0 + 1 : x1 + 1], th[ys, x0 - 1 : x1 - 1]
        else:
            th_e, th_w = np.roll(th, -1, -1)[ys, xs], np.roll(th, 1, -1)[ys, xs]
        if specified:
            th_n, th_s = th[y0 + 1 : y1 + 1, xs], th[y0 - 1 : y1 - 1, xs]
        else:
            th_n, th_s = np.roll(th, -1, -2)[ys, xs], np.roll(th, 1, -2)[ys, xs]
        thc = th[ys, xs]
        v_flux = a.v[k, ysn, xs] * (th_n + thc) - a.v[k, ys, xs] * (thc + th_s)
        u_flux = a.u[k, ys, xse] * (th_e + thc) - a.u[k, ys, xs] * (thc + th_w)
        tend = msftx * (0.5 * rdy * v_flux + 0.5 * rdx * u_flux) + m.rdnw[k] * (wdtn[k + 1] - wdtn[k])
        a.theta_work[k, ys, xs] = theta_i[k] - dts * msfty * tend


def advance_w(a, m, nl: Namelist, dts, rdx, rdy):
    """core/advance_w.py:293-627."""
    nz = a.w.shape[0] - 1
    eps_p, eps_m = 1.0 + nl.epssm, 1.0 - nl.epssm
    minv = (1.0 / m.msfty)[None]
    c1h, c2h, c1f, c2f = _col(m.c1h), _col(m.c2h), _col(m.c1f), _col(m.c2f)
    rw_tend = a.rw_tend.copy()
    w, ww, mut, muts, muave = a.w, a.ww, a.mut, a.muts, a.muave
    if nl.w_damping == 1:
        mass_f = _col(m.c1f[1:nz]) * mut[None] + _col(m.c2f[1:nz])
        safe = np.where(np.abs(mass_f) > 1.0e-12, mass_f, 1.0e-12)
        vert_cfl = np.abs(ww[1:nz] / safe * _col(m.rdnw[1:nz]) * dts)
        damp = -np.sign(w[1:nz]) * W_ALPHA * (vert_cfl - W_BETA) * mass_f
        damp = np.where(vert_cfl > W_BETA, damp, 0.0)
        rw_tend[1:nz] = rw_tend[1:nz] + damp
    mass_h = c1h * muts[None] + c2h
    t2a = (0.5 * (eps_p * a.theta_work + eps_m * a.t_2ave) + (c1h * muave[None]) * T0) / (mass_h * (T0 + a.theta_1))
    rhs = np.zeros_like(w)
    rhs[1:] = dts * (a.ph_tend[1:] + 0.5 * G * eps_m * w[1:])
    pt1 = a.ph_1 + a.phb
    wdwn = np.zeros_like(w)
    wdwn[1:] = 0.5 * (ww[1:] + ww[:-1]) * _col(m.rdnw) * (pt1[1:] - pt1[:-1])
    rhs[1:nz] = rhs[1:nz] + (-(dts * (_col(m.fnm[1:nz]) * wdwn[2:] + _col(m.fnp[1:nz]) * wdwn[1:nz])))
    mass_f_mut = c1f * mut[None] + c2f
    rhs[1:] = a.ph[1:] + m.msfty[None] * rhs[1:] / mass_f_mut[1:]
    if nl.top_lid:
        rhs[nz] = 0.0
    ht = a.phb[0] / G
    htp = np.pad(ht, ((0, 1), (0, 0)), mode="edge")
    htm = np.pad(ht, ((1, 0), (0, 0)), mode="edge")
    dy_n = htp[1:, :] - ht
    dy_s = ht - htm[:-1, :]
    htp = np.pad(ht, ((0, 0), (0, 1)), mode="edge")
    htm = np.pad(ht, ((0, 0), (1, 0)), mode="edge")
    dx_e = htp[:, 1:] - ht
    dx_w = ht - htm[:, :-1]
    cf = lambda f3: m.cf1 * f3[0] + m.cf2 * f3[1] + m.cf3 * f3[2]
    v1, u1 = a.v_1, a.u_1
    w_surface = (m.msfty * 0.5 * rdy * (dy_n * cf(v1[:3, 1:, :]) + dy_s * cf(v1[:3, :-1, :]))
                 + m.msftx * 0.5 * rdx * (dx_e * cf(u1[:3, :, 1:]) + dx_w * cf(u1[:3, :, :-1])))
    mass_h_mut = c1h * mut[None] + c2h
    smhm = np.where(np.abs(mass_h_mut) > 1.0e-12, mass_h_mut, 1.0e-12)
    coef = a.c2a * _col(m.rdnw) / smhm
    w_next = w + dts * rw_tend
    ph = a.ph
    tA_u = coef[1:nz] * (eps_p * (rhs[2 : nz + 1] - rhs[1:nz]) + eps_m * (ph[2 : nz + 1] - ph[1:nz]))
    tA_l = coef[0 : nz - 1] * (eps_p * (rhs[1:nz] - rhs[0 : nz - 1]) + eps_m * (ph[1:nz] - ph[0 : nz - 1]))
    tA = minv * a.cqw[1:nz] * (0.5 * dts * G * _col(m.rdn[1:nz])) * (tA_u - tA_l)
    buoy = a.c2a * a.alt * t2a
    tB = dts * G * minv * (_col(m.rdn[1:nz]) * (buoy[1:nz] - buoy[0 : nz - 1]) - (_col(m.c1f[1:nz]) * muave[None]))
    w_next[1:nz] = w_next[1:nz] + (tA + tB)
    km1 = nz - 1
    tA_top = (-0.5 * dts * G / smhm[km1] * m.rdnw[km1] ** 2 * 2.0 * a.c2a[km1]
              * (eps_p * (rhs[nz] - rhs[nz - 1]) + eps_m * (ph[nz] - ph[nz - 1])))
    tB_top = -dts * G * (2.0 * m.rdnw[km1] * a.c2a[km1] * a.alt[km1] * t2a[km1] + (m.c1f[nz] * muave))
    w_top = w[nz] + dts * rw_tend[nz] + minv[0] * (tA_top + tB_top)
    w_next[nz] = 0.0 if nl.top_lid else w_top
    w_next[0] = w_surface
    wf = w_next.copy()
    for k in range(1, nz + 1):
        wf[k] = (w_next[k] - a.a[k] * wf[k - 1]) * a.alpha[k]
    ws = wf.copy()
    for k in range(nz - 1, 0, -1):
        ws[k] = wf[k] - a.gamma[k] * ws[k + 1]
    if nl.damp_opt == 3 and nl.dampcoef > 0.0:
        dampmag = dts * nl.dampcoef
        hdepth = nl.zdamp
        ptd = a.ph_1 + a.phb
        htop = ptd[nz] / G
        hk = ptd / G
        hbot = (htop - hdepth)[None]
        ramp = np.sin(0.5 * np.pi * (hk - hbot) / hdepth) ** 2
        dampwt = np.where(hk >= hbot, dampmag * ramp, 0.0)
        wd = (ws - dampwt * mass_f_mut * a.w_save) / (1.0 + dampwt)
        ws[1:] = wd[1:]
    mass_f_muts = c1f * muts[None] + c2f
    ph_next = ph.copy()
    ph_next[1:] = rhs[1:] + m.msfty[None] * 0.5 * dts * G * eps_p * ws[1:] / mass_f_muts[1:]
    a.w, a.ph, a.t_2ave = ws, ph_next, t2a


def acoustic_substep(a, m, nl: Namelist, dts, bdy=None):
    """core/acoustic.py:837-1150."""
    rdx, rdy = 1.0 / nl.dx, 1.0 / nl.dy
    _, specified, nested = lateral_flags(nl)
    advance_uv(a, m, dts, rdx, rdy, nl.dx, nl.dy, nl.top_lid, bdy)
    cad = getattr(a, "cad", None)
    if cad is not None:  # ring-0 tangential winds (core/acoustic.py:777-785)
        a.u[:, 0, :] = cad.u_tan[:, 0, :]
        a.u[:, -1, :] = cad.u_tan[:, -1, :]
        a.v[:, 1:-1, 0] = cad.v_tan[:, 1:-1, 0]
        a.v[:, 1:-1, -1] = cad.v_tan[:, 1:-1, -1]
    advance_mu_t(a, m, dts, rdx, rdy, nl.epssm, specified or nested)
    if cad is not None:  # ring-0 mass and theta pins (core/acoustic.py:902-915)
        a.mu = _pin_ring(a.mu, cad.mu)
        a.muts = _pin_ring(a.muts, cad.muts)
        a.muave = _pin_ring(a.muave, cad.muave)
        a.theta_work = _pin_ring(a.theta_work, cad.theta)
    advance_w(a, m, nl, dts, rdx, rdy)
    ph_pin = getattr(a, "ph_pin", None)
    if ph_pin is not None:  # spec_bdyupdate_ph (core/acoustic.py:1059-1071)
        a.ph = _pin_ring(a.ph, ph_pin)
    if cad is not None:  # zero_grad_bdy w (core/acoustic.py:1073-1090)
        a.w = specified_w_zero_grad(a.w, a.w_save, a.mut, a.muts, m)
    mu_work = a.muts - a.mut
    al, pp = calc_al_p(mu_work, a.muts, a.ph, a.theta_work, a.theta_1, a.c2a, a.alt, m)
    a.p = pp + SMDIV * (pp - a.pm1)
    a.pm1 = pp
    a.al = al


# ----------------------------------------------------------------------------
# stage / step: runtime/operational_mode.py:1682-2265, 3319-3534
# ----------------------------------------------------------------------------

def acoustic_state_from_prep(s, prep, al0, p0, pm1, tend, carry_mudf, nl: Namelist, dts, lead_seconds,
                             bdy_relax=None, dt_rk=0.0):
    """operational_mode.py:1682-2166 (no nested forcing); with ``bdy_relax``
    the specified-domain cadence (:1984-2041): the relax ph tendency and the
    stage-end ring-0 targets."""
    m = nl.metrics
    rdx, rdy = 1.0 / nl.dx, 1.0 / nl.dy
    nz, ny, nx = s.theta.shape
    mu_prime = prep.mut - prep.mub
    if nl.moist_cqw:
        rw, cqw = pg_buoy_w_moist(s.p_perturbation, mu_prime, prep.mub, qtot_of(s), m)
    else:
        rw, cqw = pg_buoy_w_dry(s.p_perturbation, mu_prime, m)
    rw = rw + tend.w
    if nl.w_coriolis:
        c1h, c2h = _col(m.c1h), _col(m.c2h)
        ru_s = (c1h * prep.muu[None] + c2h) * s.u / m.msfuy[None]
        rv_s = (c1h * prep.muv[None] + c2h) * s.v / m.msfvx[None]
        ru_m = 0.5 * (ru_s[:, :, :-1] + ru_s[:, :, 1:])
        u_m = 0.5 * (s.u[:, :, :-1] + s.u[:, :, 1:])
        rv_m = 0.5 * (rv_s[:, :-1, :] + rv_s[:, 1:, :])
        v_m = 0.5 * (s.v[:, :-1, :] + s.v[:, 1:, :])
        fnm_f, fnp_f = _col(m.fnm[1:nz]), _col(m.fnp[1:nz])
        face = lambda f: fnm_f * f[1:nz] + fnp_f * f[: nz - 1]
        ru_f, u_f, rv_f, v_f = face(ru_m), face(u_m), face(rv_m), face(v_m)
        mxy = (m.msftx / m.msfty)[None]
        cor = m.e[None] * (m.cosa[None] * ru_f - mxy * m.sina[None] * rv_f)
        curv = W_RERADIUS * (ru_f * u_f + mxy * rv_f * v_f)
        rw[1:nz] = rw[1:nz] + (cor + curv)
    ph_tend = rhs_ph(s.u, s.v, prep.ww_save, s.ph_perturbation, prep.phb, s.w, prep.mut,
                     prep.muu, prep.muv, m, rdx, rdy, nl.top_lid, order=nl.h_sca_adv_order,
                     specified=lateral_flags(nl)[1] or lateral_flags(nl)[2])
    a = SimpleNamespace()
    a.ww = prep.ww_save.copy()
    a.ww_1 = prep.ww_save
    a.u, a.v, a.w = prep.u_work.copy(), prep.v_work.copy(), prep.w_work.copy()
    a.u_1, a.v_1 = prep.u_save, prep.v_save
    a.mu = prep.mu_save + prep.mu_work
    a.mut = prep.mut
    a.muave = np.zeros_like(prep.mu_work)
    a.muts = prep.muts.copy()
    a.muu, a.muv = prep.muu, prep.muv
    a.mudf = carry_mudf.copy()
    a.theta_1 = prep.t_save
    a.theta_tend = tend.theta
    a.mu_tend = tend.mu
    a.ph_tend = ph_tend
    a.ph = prep.ph_work.copy()
    a.p = p0
    a.pm1 = pm1
    a.al = al0
    a.t_2ave = np.zeros_like(prep.theta_work)
    a.theta_work = prep.theta_work.copy()
    a.u_tend, a.v_tend = tend.u, tend.v
    a.pb, a.alt, a.c2a, a.cqw = prep.pb, prep.alt, prep.c2a, cqw
    a.cqu, a.cqv = prep.cqu, prep.cqv
    a.phb, a.ph_1 = prep.phb, prep.ph_1
    a.w_save = prep.w_save
    a.rw_tend = rw
    a.php = prep.php
    a.cad = None
    a.ph_pin = None
    if lateral_flags(nl)[2] and lead_seconds is not None:
        # the nested child's opt-in in-loop forcings (operational_mode.py:1906-1968),
        # all from the stage state and the strips at the step's lead
        lf0 = lambda leaf: interpolate_boundary_leaf(leaf, lead_seconds, nl.update_cadence_s)
        if nl.nested_ph_relax:
            tgt = full_ring_target(lf0(s.ph_bdy), nz + 1, ny, nx)
            a.ph_tend = a.ph_tend + nested_relax_tendency(s.ph_perturbation, tgt, prep.mut, m, nl.dt_s)
        if nl.nested_w_relax:
            tgt = full_ring_target(lf0(s.w_bdy), nz + 1, ny, nx)
            a.rw_tend = a.rw_tend + nested_relax_tendency(s.w, tgt, prep.mut, m, nl.dt_s)
        if nl.nested_ph_spec:  # boundary_apply.py:1299-1340
            a.ph_pin = full_ring_target(lf0(s.ph_bdy), nz + 1, ny, nx) - prep.ph_save
    if bdy_relax is not None:
        a.ph_tend = a.ph_tend + bdy_relax.ph
        lead_stage = lead_seconds + float(dt_rk)
        lf = lambda leaf: interpolate_boundary_leaf(leaf, lead_stage, nl.update_cadence_s)
        c1h, c2h = _col(m.c1h), _col(m.c2h)
        cad = SimpleNamespace()
        cad.ph_delta = full_ring_target(lf(s.ph_bdy), nz + 1, ny, nx) - prep.ph_save
        cad.mu = full_ring_target(lf(s.mu_bdy), 1, ny, nx)[0]
        cad.muts = prep.mub + cad.mu
        cad.muave = cad.muts - prep.mut
        th_pin = full_ring_target(lf(s.theta_bdy), nz, ny, nx)
        mass_pin = c1h * cad.muts[None] + c2h
        mass_cur = c1h * prep.mut[None] + c2h
        cad.theta = mass_pin * (th_pin - T0) - mass_cur * prep.t_save
        cad.u_tan, cad.v_tan = tangential_targets(lf(s.u_bdy), lf(s.v_bdy), prep, m)
        a.cad = cad
        a.ph_pin = cad.ph_delta
    bdy = None
    if nl.run_boundary and lead_seconds is not None:
        c1h, c2h = _col(m.c1h), _col(m.c2h)
        nzone = nl.spec_zone + nl.relax_zone
        us = interpolate_boundary_leaf(s.u_bdy, lead_seconds, nl.update_cadence_s)
        vs = interpolate_boundary_leaf(s.v_bdy, lead_seconds, nl.update_cadence_s)
        bdy = SimpleNamespace()
        bdy.u_target = normal_bdy_work_target_u(us, prep.u_save, c1h * prep.muu[None] + c2h,
                                                c1h * prep.muus[None] + c2h, m.msfuy, nzone)
        bdy.v_target = normal_bdy_work_target_v(vs, prep.v_save, c1h * prep.muv[None] + c2h,
                                                c1h * prep.muvs[None] + c2h, m.msfvx, nzone)
        strength = NORMAL_BDY_RELAX_STRENGTH if nl.normal_bdy_relax_strength is None else nl.normal_bdy_relax_strength
        sub = strength * (dts / nl.dt_s if nl.dt_s != 0.0 else 0.0)
        bdy.wu = normal_relax_weights(ny, nx + 1, sub, "u")
        bdy.wv = normal_relax_weights(ny + 1, nx, sub, "v")
    return a, bdy


def small_step_finish_and_refresh(s, prep, a, nl: Namelist):
    """core/small_step_finish.py:419-498 + operational_mode.py:2169-2231."""
    m = nl.metrics
    c1h, c2h, c1f, c2f = _col(m.c1h), _col(m.c2h), _col(m.c1f), _col(m.c2f)
    ms_u = c1h * prep.muus[None] + c2h
    mc_u = c1h * prep.muu[None] + c2h
    ms_v = c1h * prep.muvs[None] + c2h
    mc_v = c1h * prep.muv[None] + c2h
    ms_w = c1f * a.muts[None] + c2f
    mc_w = c1f * prep.mut[None] + c2f
    ms_t = c1h * a.muts[None] + c2h
    mc_t = c1h * prep.mut[None] + c2h

    def sd(x):
        return np.where(np.abs(x) > 1.0e-12, x, np.where(x >= 0.0, 1.0e-12, -1.0e-12))

    n = copy_state(s)
    n.u = (m.msfuy[None] * a.u + prep.u_save * mc_u) / sd(ms_u)
    n.v = (m.msfvx[None] * a.v + prep.v_save * mc_v) / sd(ms_v)
    n.w = (m.msfty[None] * a.w + prep.w_save * mc_w) / sd(ms_w)
    n.theta = (a.theta_work + prep.t_save * mc_t) / sd(ms_t) + T0
    ph_pert = a.ph + prep.ph_save
    p_base = s.p_total - s.p_perturbation
    ph_base = s.ph_total - s.ph_perturbation
    mu_base = s.mu_total - s.mu_perturbation
    n.p_total = p_base + a.p
    n.p_perturbation = a.p
    n.ph_total = ph_base + ph_pert
    n.ph_perturbation = ph_pert
    n.mu_total = mu_base + a.mu
    n.mu_perturbation = a.mu.copy()
    # refresh grid%p (operational_mode.py:2169-2231 -> acoustic_wrf.py:322-438)
    pb = prep.pb
    phb = n.ph_total - n.ph_perturbation
    mub = prep.mub
    mhb = _col(m.c1h) * mub[None] + _col(m.c2h)
    dphb = phb[1:] - phb[:-1]
    den = _col(m.dnw) * mhb
    alb = -dphb / np.where(np.abs(den) > 1.0e-12, den, 1.0e-12)
    muts = mub + n.mu_perturbation
    mw = _col(m.c1h) * muts[None] + _col(m.c2h)
    smw = np.where(np.abs(mw) > 1.0e-12, mw, 1.0e-12)
    php_ = n.ph_perturbation
    if nl.hypsometric_opt == 2:
        dph_tot = (phb[1:] + php_[1:]) - (phb[:-1] + php_[:-1])
        alb_used = _log_alpha(phb[1:] - phb[:-1], mub[None], m)
        al = _log_alpha(dph_tot, muts[None], m) - alb_used
    else:
        al = -(alb * _col(m.c1h) * n.mu_perturbation[None] + _col(m.rdnw) * (php_[1:] - php_[:-1])) / smw
        alb_used = alb
    alt = al + alb_used
    p_pert = pressure_from_theta_alt(n.theta, alt) - pb
    p_base2 = n.p_total - n.p_perturbation
    n.p_total = p_base2 + p_pert
    n.p_perturbation = p_pert
    return n


def rk_scan_step(carry, nl: Namelist, lead_seconds=None, physics=None):
    """``_rk_scan_step`` (operational_mode.py:3319-3534).

    ``carry`` is a SimpleNamespace with ``state`` and ``mudf``; the returned
    carry adds t_2ave, ww, mudf, muave, muts, ph_tend and the *_save family.
    ``physics`` (DryPhysicsTendencies attributes) is merged into every stage's
    tendencies by ``rk_addtend_dry``.
    """
    m = nl.metrics
    rdx, rdy = 1.0 / nl.dx, 1.0 / nl.dy
    origin = copy_state(carry.state)
    dt = float(nl.dt_s)
    ns = int(nl.acoustic_substeps)
    stages = ((1, dt / 3.0, dt / 3.0, 1), (2, 0.5 * dt, dt / float(ns), max(1, ns // 2)), (3, dt, dt / float(ns), ns))
    _, specified, nested = lateral_flags(nl)
    moist = nl.moist_adv_opt != 0
    # the specified-domain boundary cadence (operational_mode.py:2478-2530, 3362)
    bdy_relax = None
    if nl.specified_bdy_cadence and specified and lead_seconds is not None:
        bdy_relax = specified_relax_dry_tendencies(origin, lead_seconds, m, dt, nl.update_cadence_s)
    state = origin
    mudf = carry.mudf.copy()
    out = SimpleNamespace()
    for rk_step, dt_rk, dts, nsub in stages:
        s = state
        vel = couple_velocities_periodic(s.u, s.v, s.mu_total, m, rdx, rdy)
        if nl.specified_adv_degrade and specified:  # operational_mode.py:2464-2475, 2494-2507
            vel.specified = True
            vel.ru_full, vel.rv_full = couple_uv_specified(s.u, s.v, s.mu_total, m)
        tend = augment_large_step_tendencies(s, origin, vel, nl, rk_step, bdy_relax, physics)
        q_tend = moisture_coupled_tendencies(s, origin, vel, nl, rk_step) if moist else None
        ww_stage = stage_omega_specified(s.u, s.v, s.mu_total, m, rdx, rdy) if (specified or nested) else vel.rom
        prep = small_step_prep(s, origin, rk_step, m, ww_stage)
        al0, p0 = calc_al_p(prep.mu_work, prep.muts, prep.ph_work, prep.theta_work, prep.theta_1, prep.c2a, prep.alt, m)
        a, bdy = acoustic_state_from_prep(s, prep, al0, p0, p0.copy(), tend, mudf, nl, dts, lead_seconds,
                                          bdy_relax, dt_rk)
        a.a, a.alpha, a.gamma = calc_coef_w(prep.mut, m, dts, nl.epssm, nl.top_lid, a.cqw, prep.c2a)
        for _ in range(nsub):
            acoustic_substep(a, m, nl, dts, bdy)
        n = small_step_finish_and_refresh(s, prep, a, nl)
        if moist:
            mo = _col(m.c1h) * origin.mu_total[None] + _col(m.c2h)
            mn = _col(m.c1h) * n.mu_total[None] + _col(m.c2h)
            inv = 1.0 / mn
            for name, qt in zip(MOIST_SPECIES, q_tend):
                setattr(n, name, (mo * getattr(origin, name) + dt_rk * qt) * inv)
        state = n
        mudf = a.mudf
        out.t_2ave = a.t_2ave + T0
        out.ww = a.ww + prep.ww_save
        out.muave = a.muave
        out.muts = a.muts
        out.ph_tend = a.ph_tend
        out.u_save, out.v_save, out.w_save = prep.u_save, prep.v_save, prep.w_save
        out.t_save = prep.t_save + T0
        out.ph_save = prep.ph_save
        out.mu_save = prep.mu_save
        out.ww_save = prep.ww_save
    out.state = state
    out.mudf = mudf
    return out


def stage_acoustic_state(carry, nl: Namelist, rk_step: int = 3, lead_seconds=None):
    """The acoustic work state and stage constants that ``rk_scan_step`` hands
    its small-step loop (operational_mode.py:1682-2166), for RK stage
    ``rk_step`` entered from ``carry.state`` (used as both the stage and the
    step-start state), without the specified-domain cadence and the nested
    forcings.  Returns ``(a, dts, s, bdy)``: ``a`` as ``acoustic_substep``
    takes it, the substep length, the stage state and the boundary relaxation
    (None unless run_boundary with a lead).  Test infrastructure for the
    substep operator and its adjoint."""
    m = nl.metrics
    rdx, rdy = 1.0 / nl.dx, 1.0 / nl.dy
    s = copy_state(carry.state)
    dt = float(nl.dt_s)
    ns = int(nl.acoustic_substeps)
    dt_rk, dts = {1: (dt / 3.0, dt / 3.0), 2: (0.5 * dt, dt / float(ns)), 3: (dt, dt / float(ns))}[rk_step]
    _, specified, nested = lateral_flags(nl)
    vel = couple_velocities_periodic(s.u, s.v, s.mu_total, m, rdx, rdy)
    tend = augment_large_step_tendencies(s, s, vel, nl, rk_step, None)
    ww_stage = stage_omega_specified(s.u, s.v, s.mu_total, m, rdx, rdy) if (specified or nested) else vel.rom
    prep = small_step_prep(s, s, rk_step, m, ww_stage)
    al0, p0 = calc_al_p(prep.mu_work, prep.muts, prep.ph_work, prep.theta_work, prep.theta_1, prep.c2a, prep.alt, m)
    a, bdy = acoustic_state_from_prep(s, prep, al0, p0, p0.copy(), tend, carry.mudf, nl, dts, lead_seconds, None,
                                      dt_rk)
    a.a, a.alpha, a.gamma = calc_coef_w(prep.mut, m, dts, nl.epssm, nl.top_lid, a.cqw, prep.c2a)
    return a, dts, s, bdy


# ---- end-of-step lateral boundaries (coupling/boundary_apply.py:154-326, 503-663) ----

def _relax_row(field, forcing, side, b, z_len, side_len, wf, wg):
    """boundary_apply.py:589-640: the relaxed row b of one side, from the
    unmodified field and the leaf strips b-1, b, b+1 (tangential clamp)."""
    if side == "W":
        cur, te, ti = field[:, :, b], field[:, :, b - 1], field[:, :, b + 1]
    elif side == "E":
        x = field.shape[2] - 1 - b
        cur, te, ti = field[:, :, x], field[:, :, x + 1], field[:, :, x - 1]
    elif side == "S":
        cur, te, ti = field[:, b, :], field[:, b - 1, :], field[:, b + 1, :]
    else:
        y = field.shape[1] - 1 - b
        cur, te, ti = field[:, y, :], field[:, y + 1, :], field[:, y - 1, :]
    fls0 = _strip(forcing, side, b, z_len, side_len) - cur
    fls1 = _shift_clamp(fls0, +1, 1)
    fls2 = _shift_clamp(fls0, -1, 1)
    fls3 = _strip(forcing, side, b - 1, z_len, side_len) - te
    fls4 = _strip(forcing, side, b + 1, z_len, side_len) - ti
    lap = fls1 + fls2 + fls3 + fls4 - 4.0 * fls0
    return cur + wf * fls0 - wg * lap


def _apply_side_spec(field, forcing, side, spec_zone=1):
    """boundary_apply.py:556-570: the outer spec_zone rows set to the strips."""
    z_len, y_len, x_len = field.shape
    out = field.copy()
    for b in range(spec_zone):
        if side == "W":
            out[:, :, b] = _strip(forcing, side, b, z_len, y_len)
        elif side == "E":
            out[:, :, x_len - 1 - b] = _strip(forcing, side, b, z_len, y_len)
        elif side == "S":
            out[:, b, :] = _strip(forcing, side, b, z_len, x_len)
        else:
            out[:, y_len - 1 - b, :] = _strip(forcing, side, b, z_len, x_len)
    return out


def lbc_apply_3d(field, leaf, lead_seconds, dt_s, cadence, spec_zone=1, relax_zone=4):
    """boundary_apply.py:503-525 (+ :622-663): every side's relax rows from the
    unmodified field (W / E columns trimmed to rows [b+1, y_len-b-2], S / N
    rows to columns [b, x_len-b-1]), then the spec rows (W, E, S, N)."""
    forcing = interpolate_boundary_leaf(leaf, lead_seconds, cadence)
    z_len, y_len, x_len = field.shape
    out = field.copy()
    for side in SIDES:
        for b in range(spec_zone, relax_zone):
            wf, wg = _wrf_relax_weights(b, dt_s, spec_zone, relax_zone)
            if side in ("W", "E"):
                row = _relax_row(field, forcing, side, b, z_len, y_len, wf, wg)
                col = b if side == "W" else x_len - 1 - b
                out[:, b + 1:y_len - b - 1, col] = row[:, b + 1:y_len - b - 1]
            else:
                row = _relax_row(field, forcing, side, b, z_len, x_len, wf, wg)
                r = b if side == "S" else y_len - 1 - b
                out[:, r, b:x_len - b] = row[:, b:x_len - b]
    for side in SIDES:
        out = _apply_side_spec(out, forcing, side, spec_zone)
    return out


def lbc_apply_3d_spec_only(field, leaf, lead_seconds, cadence, spec_zone=1):
    """boundary_apply.py:154-167: the spec rows only."""
    forcing = interpolate_boundary_leaf(leaf, lead_seconds, cadence)
    out = field
    for side in SIDES:
        out = _apply_side_spec(out, forcing, side, spec_zone)
    return out


def apply_lateral_boundaries(s, lead_seconds, dt_s, nl: Namelist, dry_spec_only=False):
    """``apply_lateral_boundaries`` (coupling/boundary_apply.py:170-326) on an
    oracle state carrying the ``*_bdy`` leaves (u, v, w, theta, qv..qg, p, pb,
    mu, mub, ph, phb); the moisture leaves are optional (absent: untouched)."""
    cad = nl.update_cadence_s
    a3 = lambda f, leaf: lbc_apply_3d(f, leaf, lead_seconds, dt_s, cad, nl.spec_zone, nl.relax_zone)
    s3 = lambda f, leaf: lbc_apply_3d_spec_only(f, leaf, lead_seconds, cad, nl.spec_zone)
    n = copy_state(s)
    for q in MOIST_SPECIES:
        leaf = getattr(s, q + "_bdy", None)
        if leaf is not None:
            setattr(n, q, np.maximum(a3(getattr(s, q), leaf), 0.0))
    mub0 = (s.mu_total - s.mu_perturbation)[None]
    phb0 = s.ph_total - s.ph_perturbation
    if dry_spec_only:
        n.u, n.v, n.theta = s3(s.u, s.u_bdy), s3(s.v, s.v_bdy), s3(s.theta, s.theta_bdy)
        mu_p = s3(s.mu_perturbation[None], s.mu_bdy)[0]
        mub = s3(mub0, s.mub_bdy)[0]
        ph_p = s3(s.ph_perturbation, s.ph_bdy)
        phb = s3(phb0, s.phb_bdy)
        n.ph_total, n.ph_perturbation = phb + ph_p, ph_p
        n.mu_total, n.mu_perturbation = mub + mu_p, mu_p
        return n
    n.u, n.v, n.w, n.theta = a3(s.u, s.u_bdy), a3(s.v, s.v_bdy), a3(s.w, s.w_bdy), a3(s.theta, s.theta_bdy)
    p_p = a3(s.p_perturbation, s.p_bdy)
    pb = a3(s.p_total - s.p_perturbation, s.pb_bdy)
    mu_p = a3(s.mu_perturbation[None], s.mu_bdy)[0]
    mub = a3(mub0, s.mub_bdy)[0]
    if nl.force_geopotential:
        ph_p = a3(s.ph_perturbation, s.ph_bdy)
        phb = a3(phb0, s.phb_bdy)
        n.ph_total, n.ph_perturbation = phb + ph_p, ph_p
    n.p_total, n.p_perturbation = pb + p_p, p_p
    n.mu_total, n.mu_perturbation = mub + mu_p, mu_p
    return n


# ----------------------------------------------------------------------------
# post-step guards (runtime/operational_mode.py:1300-1520, 4950-4983)
# ----------------------------------------------------------------------------

THETA_LIMITER_MIN_K = 0.0     # operational_mode.py:180
THETA_LIMITER_MAX_K = 1000.0  # operational_mode.py:198
MIXING_RATIO_MAX = 0.05       # operational_mode.py:1300


def valid_mixing_ratio(candidate, origin, upper=MIXING_RATIO_MAX):
    """``_valid_mixing_ratio`` (operational_mode.py:1300-1306)."""
    c = np.asarray(candidate, dtype=np.float64)
    with np.errstate(invalid="ignore"):
        ok = np.isfinite(c) & (c >= 0.0) & (c <= upper)
    return np.where(ok, c, origin)


def finite_or_origin(candidate, origin):
    """``_finite_or_origin`` (operational_mode.py:1309-1314)."""
    c = np.asarray(candidate, dtype=np.float64)
    return np.where(np.isfinite(c), c, origin)


def theta_mass_weights(theta, mu_total):
    """``_theta_mass_weights`` (operational_mode.py:1317-1323)."""
    m = np.asarray(mu_total, dtype=np.float64)
    with np.errstate(invalid="ignore"):
        m = np.where(np.isfinite(m) & (m > 0.0), m, 0.0)
    return np.broadcast_to(m[None], np.shape(theta))


def first_limited_cell_xyz(mask):
    """``_first_limited_cell_xyz`` (operational_mode.py:1342-1357): the first
    True cell in (z, y, x) order as [x, y, z], or [-1, -1, -1]."""
    flat = np.flatnonzero(np.ravel(mask))
    if flat.size == 0:
        return np.array([-1, -1, -1], dtype=np.int32)
    z, rem = divmod(int(flat[0]), mask.shape[1] * mask.shape[2])
    y, x = divmod(rem, mask.shape[2])
    return np.array([x, y, z], dtype=np.int32)


def empty_theta_limiter_diagnostics():
    """``_empty_theta_limiter_diagnostics`` (operational_mode.py:1374-1384)."""
    return {"theta_limited_cell_count": 0, "theta_first_limited_cell_xyz": np.array([-1, -1, -1], dtype=np.int32),
            "theta_mass_before": 0.0, "theta_mass_after": 0.0, "theta_mass_residual": 0.0}


def theta_increment_limiter(candidate, origin, mass, minimum_k=THETA_LIMITER_MIN_K, maximum_k=THETA_LIMITER_MAX_K,
                            lower_bound=None, upper_bound=None):
    """``_positive_definite_theta_increment_limiter`` (operational_mode.py:
    1387-1455): offending cells (non-finite, above ``upper`` or below
    ``lower``) keep the RK direction with the increment scaled into the
    interval; the removed mass-weighted increment is spread over every cell in
    proportion to its room, so the domain integral of theta * mass is kept."""
    c = np.asarray(candidate, dtype=np.float64)
    o = np.asarray(origin, dtype=np.float64)
    m = np.asarray(mass, dtype=np.float64)
    lower = np.float64(minimum_k)
    upper = np.float64(maximum_k)
    if lower_bound is not None:
        lower = np.maximum(lower, np.asarray(lower_bound, dtype=np.float64))
    if upper_bound is not None:
        upper = np.minimum(upper, np.asarray(upper_bound, dtype=np.float64))
    upper = np.maximum(upper, lower)
    mid = 0.5 * (lower + upper)
    safe_o = np.where(np.isfinite(o), o, mid)
    safe_o = np.minimum(np.maximum(safe_o, lower), upper)
    fc = np.where(np.isfinite(c), c, safe_o)
    raw = fc - safe_o
    mask = ~np.isfinite(c) | (fc > upper) | (fc < lower)
    pos, neg = raw > 0.0, raw < 0.0
    ua = (upper - safe_o) / np.where(pos, raw, 1.0)
    la = (lower - safe_o) / np.where(neg, raw, -1.0)
    alpha = np.where(pos, ua, np.where(neg, la, 1.0))
    alpha = np.where(mask, np.minimum(np.maximum(alpha, 0.0), 1.0), 1.0)
    lim0 = safe_o + alpha * raw
    target = np.sum(fc * m)
    mass0 = np.sum(lim0 * m)
    residual = target - mass0
    room = np.where(residual >= 0.0, upper - lim0, lim0 - lower)
    cap = np.sum(room * m)
    frac = min(abs(residual) / cap, 1.0) if cap > 0.0 else 0.0
    lim = lim0 + np.sign(residual) * frac * room
    lim = np.minimum(np.maximum(lim, lower), upper)
    after = np.sum(lim * m)
    diag = {"theta_limited_cell_count": int(mask.sum()), "theta_first_limited_cell_xyz": first_limited_cell_xyz(mask),
            "theta_mass_before": float(target), "theta_mass_after": float(after),
            "theta_mass_residual": float(after - target)}
    return lim, diag


def limit_guarded_mass_state(candidate, origin):
    """``_limit_guarded_mass_state`` (operational_mode.py:1458-1470): dry mass
    that is non-finite or below 1 Pa falls back to the origin's (total and
    perturbation together)."""
    mt, mp = np.asarray(candidate.mu_total), np.asarray(candidate.mu_perturbation)
    with np.errstate(invalid="ignore"):
        ok = np.isfinite(mt) & np.isfinite(mp) & (mt >= 1.0)
    n = copy_state(candidate)
    n.mu_total = np.where(ok, mt, origin.mu_total)
    n.mu_perturbation = np.where(ok, mp, origin.mu_perturbation)
    return n


def limit_guarded_dynamics_state(candidate, origin):
    """``_limit_guarded_dynamics_state_with_diagnostics`` (operational_mode.py:
    1473-1512): the theta limiter weighted by the candidate's column mass, then
    the dry-mass guard."""
    mass = theta_mass_weights(candidate.theta, candidate.mu_total)
    theta, diag = theta_increment_limiter(candidate.theta, origin.theta, mass)
    n = copy_state(candidate)
    n.theta = theta
    return limit_guarded_mass_state(n, origin), diag


def step_epilogue(next_state, origin, lead_seconds, dt_s, nl, run_boundary, disable_guards=False,
                  dry_spec_only=False):
    """The forecast step after ``_rk_scan_step`` without physics
    (operational_mode.py:4950-4983): the dynamics guards (theta limiter,
    dry-mass guard, every moisture species checked against the origin), the
    end-of-step lateral boundary pass, then the finite / mixing-ratio /
    dry-mass guards of the bounded state.  Returns (state, diagnostics)."""
    s, diag = next_state, empty_theta_limiter_diagnostics()
    if not disable_guards:
        s, diag = limit_guarded_dynamics_state(s, origin)
        for q in MOIST_SPECIES:
            setattr(s, q, valid_mixing_ratio(getattr(s, q), getattr(origin, q)))
    if run_boundary:
        b = apply_lateral_boundaries(s, lead_seconds, dt_s, nl, dry_spec_only=dry_spec_only)
        if disable_guards:
            s = b
        else:
            s = copy_state(b)
            for f in ("u", "v", "w", "theta", "p_total", "ph_total", "p_perturbation", "ph_perturbation"):
                setattr(s, f, finite_or_origin(getattr(b, f), getattr(origin, f)))
            s.qv = valid_mixing_ratio(b.qv, origin.qv)
            s = limit_guarded_mass_state(s, origin)
    return s, diag
