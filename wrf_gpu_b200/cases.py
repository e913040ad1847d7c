"""Synthetic input builders for the dycore step workloads (host NumPy, float64).

These build the reference's data contract -- ``DycoreMetrics``
(``src/gpuwrf/contracts/grid.py:66-240``), ``State`` leaves
(``contracts/state.py:82-206``) and the step controls of ``OperationalNamelist``
(``runtime/operational_mode.py:410-700``) -- for seeded synthetic workloads of
the shapes the benchmarks are quoted on.  The initial-condition procedure
follows the reference's idealized builder (``ic_generators/idealized.py``):
a hydrostatic base column integrated with the discrete WRF relation
``phb(k+1) = phb(k) - dnw(k)*(c1h*mub+c2h)*alb(k)``, a fixed-mass hydrostatic
rebalance of the perturbation geopotential after the theta perturbation
(``idealized.py:440-490``) and the perturbation pressure diagnosed from the
equation of state (``idealized.py:492-541``).

Nothing here runs on the hot path; it only prepares inputs.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from types import SimpleNamespace

import numpy as np

R_D = 287.0
CP_D = 7.0 * R_D / 2.0
P0 = 100000.0
G = 9.81
CPOVCV = CP_D / (CP_D - R_D)
CVPM = -(CP_D - R_D) / CP_D
MOIST = ("qv", "qc", "qr", "qi", "qs", "qg")


def flat_metrics(eta: np.ndarray, ny: int, nx: int, p_top: float, *, c3_placeholder: bool = False):
    """``DycoreMetrics.flat`` (``contracts/grid.py:170-240``) with the pure-sigma
    override of the idealized grid (``ic_generators/idealized.py:416-438``):
    c1h = c1f = 1, c2h = c2f = 0.  ``c3*`` are the eta levels (so the log
    hypsometric form is usable) unless ``c3_placeholder`` reproduces the
    idealized placeholder c3 = 1, c4 = 0."""
    eta = np.asarray(eta, dtype=np.float64)
    nz = eta.size - 1
    if nz < 4:
        raise ValueError("nz >= 4 required")
    dnw = eta[1:] - eta[:-1]
    rdnw = 1.0 / dnw
    dn = np.ones(nz)
    dn[1:] = 0.5 * (dnw[1:] + dnw[:-1])
    dn[0] = dnw[0]
    rdn = 1.0 / dn
    fnm = np.zeros(nz)
    fnp = np.zeros(nz)
    fnp[1:] = 0.5 * dnw[1:] / dn[1:]
    fnm[1:] = 0.5 * dnw[:-1] / dn[1:]
    cof1 = (2.0 * dn[1] + dn[2]) / (dn[1] + dn[2]) * dnw[0] / dn[1]
    cof2 = dn[1] / (dn[1] + dn[2]) * dnw[0] / dn[2]
    eta_mass = 0.5 * (eta[:-1] + eta[1:])
    m = SimpleNamespace(
        msftx=np.ones((ny, nx)), msfty=np.ones((ny, nx)),
        msfux=np.ones((ny, nx + 1)), msfuy=np.ones((ny, nx + 1)),
        msfvx=np.ones((ny + 1, nx)), msfvy=np.ones((ny + 1, nx)),
        c1h=np.ones(nz), c2h=np.zeros(nz), c1f=np.ones(nz + 1), c2f=np.zeros(nz + 1),
        c3h=np.ones(nz) if c3_placeholder else eta_mass.copy(), c4h=np.zeros(nz),
        c3f=np.ones(nz + 1) if c3_placeholder else eta.copy(), c4f=np.zeros(nz + 1),
        dn=dn, dnw=dnw, rdn=rdn, rdnw=rdnw, fnm=fnm, fnp=fnp,
        cf1=float(fnp[1] + cof1), cf2=float(fnm[1] - cof1 - cof2), cf3=float(cof2),
        f=np.zeros((ny, nx)), e=np.zeros((ny, nx)), sina=np.zeros((ny, nx)), cosa=np.ones((ny, nx)),
        p_top=float(p_top), eta=eta,
    )
    return m


def _alpha(theta, p):
    """Dry specific volume from the EOS used by the dycore."""
    return (R_D / P0) * theta * ((p / P0) ** CVPM)


@dataclass
class Case:
    """A complete step input: metrics, namelist controls, initial state."""

    name: str
    nx: int
    ny: int
    nz: int
    metrics: SimpleNamespace
    controls: dict
    state: SimpleNamespace
    mudf: np.ndarray
    notes: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def _balanced_state(m, theta_full, theta_base, mub, ht, u, v, moist=None):
    """Hydrostatic base + fixed-mass rebalance (``idealized.py:440-541``), per column.

    ``theta_full``/``theta_base`` are (nz, ny, nx); ``mub``/``ht`` (ny, nx).
    Pure sigma: ``p_hyd = eta_mass*mub + p_top``, mass weight ``c1h*mub + c2h``.
    """
    nz, ny, nx = theta_full.shape
    eta = m.eta
    eta_mass = 0.5 * (eta[:-1] + eta[1:])
    pb = eta_mass[:, None, None] * mub[None] + m.p_top
    alb = _alpha(theta_base, pb)
    alt_full = _alpha(theta_full, pb)
    al = alt_full - alb
    mass_h = m.c1h[:, None, None] * mub[None] + m.c2h[:, None, None]
    phb = np.zeros((nz + 1, ny, nx))
    php = np.zeros((nz + 1, ny, nx))
    phb[0] = G * ht
    for k in range(nz):
        phb[k + 1] = phb[k] - m.dnw[k] * mass_h[k] * alb[k]
        php[k + 1] = php[k] - m.dnw[k] * mass_h[k] * al[k]
    al_diag = -(m.rdnw[:, None, None] * (php[1:] - php[:-1])) / mass_h
    alt_diag = al_diag + alb
    p_full = P0 * ((R_D * theta_full) / (P0 * alt_diag)) ** CPOVCV
    p_pert = p_full - pb
    s = SimpleNamespace(
        u=u, v=v, w=np.zeros((nz + 1, ny, nx)), theta=theta_full.copy(),
        p_total=pb + p_pert, p_perturbation=p_pert,
        ph_total=phb + php, ph_perturbation=php,
        mu_total=mub.copy(), mu_perturbation=np.zeros((ny, nx)),
    )
    for name in MOIST:
        setattr(s, name, np.zeros((nz, ny, nx)) if moist is None else moist[name])
    return s


def _controls(**kw):
    base = dict(dt_s=10.0, acoustic_substeps=10, epssm=0.1, top_lid=False, w_damping=0, damp_opt=0,
                dampcoef=0.0, zdamp=5000.0, hypsometric_opt=1, h_sca_adv_order=2, scalar_adv_opt=0,
                moist_adv_opt=0, run_boundary=False, bc_ideal=True, spec_zone=1, relax_zone=4,
                update_cadence_s=3600.0, normal_bdy_relax_strength=None, moist_cqw=True, w_coriolis=True)
    base.update(kw)
    return base


def _boundary_leaves(state, nz, ny, nx, times=2, width=5, rng=None, full=False):
    """Specified boundary strips ``(time, side, width, z, side_len)`` (``contracts/state.py:96-106``)
    of u, v, theta (full), ph' (nz+1 levels), mu' (one level) and w (nz+1
    levels), built from the initial edge rows: constant in time, or with
    ``rng`` perturbed by seeded noise and drifting between the two time levels
    (u/v 0.5 m/s, theta 0.3 K, ph' 20 m2/s2, mu' 30 Pa, w 0.2 m/s).  With
    ``full`` also the strips the end-of-step lateral boundary pass reads
    (``coupling/boundary_apply.py:170-326``): p', pb, mub, phb and the six
    mixing ratios, from the same edge rows (unperturbed)."""
    side = max(nx + 1, ny + 1)
    out = {}
    specs = (("u_bdy", state.u, 0.5), ("v_bdy", state.v, 0.5), ("theta_bdy", state.theta, 0.3),
             ("ph_bdy", state.ph_perturbation, 20.0), ("mu_bdy", state.mu_perturbation[None], 30.0),
             ("w_bdy", state.w, 0.2))
    if full:
        specs = specs + (("p_bdy", state.p_perturbation, 0.0), ("pb_bdy", state.p_total - state.p_perturbation, 0.0),
                         ("mub_bdy", (state.mu_total - state.mu_perturbation)[None], 0.0),
                         ("phb_bdy", state.ph_total - state.ph_perturbation, 0.0)) + \
            tuple((q + "_bdy", getattr(state, q), 0.0) for q in MOIST)
    for name, fld, scale in specs:
        zl, yl, xl = fld.shape
        leaf = np.zeros((times, 4, width, zl, side))
        for b in range(width):
            leaf[:, 0, b, :, :yl] = fld[:, :, b]
            leaf[:, 1, b, :, :yl] = fld[:, :, xl - 1 - b]
            leaf[:, 2, b, :, :xl] = fld[:, b, :]
            leaf[:, 3, b, :, :xl] = fld[:, yl - 1 - b, :]
        if rng is not None and scale > 0.0:
            leaf = leaf + scale * rng.standard_normal(leaf.shape[1:])[None]
            leaf[1:] = leaf[1:] + 0.5 * scale * rng.standard_normal(leaf[1:].shape)
        out[name] = leaf
    return out


def warm_bubble_3d(nx: int = 64, ny: int = 64, nz: int = 40, *, dx: float = 1000.0, ztop: float = 20000.0,
                   dt: float = 6.0, ns: int = 6) -> Case:
    """Dry 3-D warm bubble: isentropic 300 K, ps = 1000 hPa, uniform eta, flat,
    +2 K cos^2 bubble (radius 2 km, centred at the domain centre, z = 2 km),
    no wind, doubly periodic, rigid lid, dt 6 s with 6 acoustic substeps."""
    theta0 = 300.0
    exner_top = 1.0 - G * ztop / (CP_D * theta0)
    p_top = P0 * exner_top ** (CP_D / R_D)
    eta = np.linspace(1.0, 0.0, nz + 1)
    m = flat_metrics(eta, ny, nx, p_top)
    mub = np.full((ny, nx), P0 - p_top)
    ht = np.zeros((ny, nx))
    eta_mass = 0.5 * (eta[:-1] + eta[1:])
    pb1 = eta_mass * (P0 - p_top) + p_top
    z_mass = CP_D * theta0 / G * (1.0 - (pb1 / P0) ** (R_D / CP_D))
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    xc, yc = 0.5 * nx * dx, 0.5 * ny * dx
    r = np.sqrt(((x[None, None, :] - xc) / 2000.0) ** 2 + ((y[None, :, None] - yc) / 2000.0) ** 2
                + ((z_mass[:, None, None] - 2000.0) / 2000.0) ** 2)
    bubble = np.where(r <= 1.0, 2.0 * np.cos(0.5 * np.pi * r) ** 2, 0.0)
    theta_base = np.full((nz, ny, nx), theta0)
    s = _balanced_state(m, theta_base + bubble, theta_base, mub, ht,
                        np.zeros((nz, ny, nx + 1)), np.zeros((nz, ny + 1, nx)))
    c = _controls(dt_s=dt, acoustic_substeps=ns, epssm=0.1, top_lid=True)
    return Case("warm_bubble_3d", nx, ny, nz, m, dict(c, dx=dx, dy=dx), s, np.zeros((ny, nx)),
                notes={"p_top": p_top, "z_mass": z_mass})


def warm_bubble_2d() -> Case:
    """The reference's own 2-D Skamarock warm bubble (``idealized.py:195-276, 566-602``):
    80 x 1 x 40, dx = dz = 250 m, uniform-z eta-hydrostatic base, dt = 0.1 s,
    10 substeps, rigid lid, w_damping = 1, damp_opt = 3 (dampcoef 0.2, zdamp 3 km).
    Uses the builder's own cp = 1004 for the initial condition, as the reference does."""
    cp_ic = 1004.0
    cv_ic = cp_ic - R_D
    dx = dz = 250.0
    nx, nz = 80, 40
    x_m = (np.arange(nx) + 0.5) * dx
    z_m = (np.arange(nz) + 0.5) * dz
    z_face = np.arange(nz + 1) * dz

    def alpha_ic(theta, p):
        return (R_D / P0) * theta * (p / P0) ** (-cv_ic / cp_ic)

    p_face = np.zeros(nz + 1)
    p_face[0] = P0
    for k in range(nz):
        d = z_face[k + 1] - z_face[k]
        a_lo = alpha_ic(300.0, p_face[k])
        p_mid = p_face[k] - 0.5 * G * d / a_lo
        a_mid = alpha_ic(300.0, p_mid)
        p_face[k + 1] = p_face[k] - G * d / a_mid
    p_top = float(p_face[-1])
    mu = float(p_face[0] - p_top)
    eta = (p_face - p_top) / mu
    p_mass = 0.5 * (p_face[:-1] + p_face[1:])
    xx, zz = np.meshgrid(x_m, z_m)
    radius = np.sqrt(((xx - 10000.0) / 2000.0) ** 2 + ((zz - 2000.0) / 2000.0) ** 2)
    tp = 2.0 * np.where(radius <= 1.0, 0.5 * (1.0 + np.cos(np.pi * radius)), 0.0)
    tp *= 2.0 / float(np.max(tp))
    theta_k = 300.0 + tp
    m = flat_metrics(eta, 1, nx, p_top, c3_placeholder=True)
    wrf_dnw = eta[1:] - eta[:-1]
    alt_full = alpha_ic(theta_k, p_mass[:, None])
    alb = alpha_ic(np.full(nz, 300.0), p_mass)
    al = alt_full - alb[:, None]
    phb = np.zeros(nz + 1)
    php = np.zeros((nz + 1, nx))
    for k in range(nz):
        phb[k + 1] = phb[k] - wrf_dnw[k] * mu * alb[k]
        php[k + 1] = php[k] - wrf_dnw[k] * mu * al[k]
    al_diag = -((1.0 / wrf_dnw)[:, None] * (php[1:] - php[:-1])) / mu
    alt_diag = al_diag + alb[:, None]
    p_full = P0 * ((R_D * theta_k) / (P0 * alt_diag)) ** (cp_ic / cv_ic)
    p_pert = p_full - p_mass[:, None]
    s = SimpleNamespace(
        u=np.zeros((nz, 1, nx + 1)), v=np.zeros((nz, 2, nx)), w=np.zeros((nz + 1, 1, nx)),
        theta=theta_k[:, None, :].copy(),
        p_total=(p_mass[:, None] + p_pert)[:, None, :], p_perturbation=p_pert[:, None, :],
        ph_total=(phb[:, None] + php)[:, None, :], ph_perturbation=php[:, None, :],
        mu_total=np.full((1, nx), mu), mu_perturbation=np.zeros((1, nx)),
    )
    for name in MOIST:
        setattr(s, name, np.zeros((nz, 1, nx)))
    c = _controls(dt_s=0.1, acoustic_substeps=10, epssm=0.1, top_lid=True, w_damping=1, damp_opt=3,
                  dampcoef=0.2, zdamp=3000.0)
    return Case("warm_bubble_2d", nx, 1, nz, m, dict(c, dx=dx, dy=dx), s, np.zeros((1, nx)),
                notes={"x_m": x_m, "z_m": z_m})


def _spectral_terrain(ny, nx, hmax, seed, kcut=0.05):
    """Seeded random field with power ~ k^-2, tapered by exp(-(k/kcut)^2) (k in
    cycles per grid point; kcut 0.05 keeps wavelengths >~ 20 dx, the smoothing a
    terrain-following grid needs), rescaled to 0..hmax."""
    rng = np.random.default_rng(seed)
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    k = np.sqrt(kx ** 2 + ky ** 2)
    k[0, 0] = 1.0
    amp = k ** (-1.0) * np.exp(-((k / kcut) ** 2))
    amp[0, 0] = 0.0
    spec = amp * (rng.standard_normal(amp.shape) + 1j * rng.standard_normal(amp.shape))
    h = np.fft.irfft2(spec, s=(ny, nx))
    h = (h - h.min()) / max(h.max() - h.min(), 1e-30)
    return hmax * h


def _qsat(t, p):
    es = 611.2 * np.exp(17.67 * (t - 273.15) / (t - 29.65))
    return 0.622 * es / np.maximum(p - es, 1.0)


def real_like_moist(nx: int = 433, ny: int = 433, nz: int = 50, *, seed: int = 0, dx: float = 1000.0,
                    ztop: float = 20000.0, dt: float = 6.0, ns: int = 6, hmax: float = 3000.0,
                    specified: bool = True, bdy_noise: bool = False) -> Case:
    """Real-like moist synthetic: seeded k^-2 spectral terrain (0..hmax), theta from 295 K
    at the surface with N = 0.011 1/s, seeded 5->20 m/s shear plus N(0, 0.5^2) white noise
    on u/v, qv at 80 % RH decaying with height, lognormal qc/qr in 2-6 km.  Specified
    lateral boundaries (constant-in-time strips; with ``bdy_noise`` seeded
    perturbed strips that drift in time), moist_adv_opt = 1 (positive definite),
    dt 6 s, 6 acoustic substeps, epssm 0.1, no lid."""
    rng = np.random.default_rng(seed + 1)
    theta_s, nbv = 295.0, 0.011
    theta0 = 300.0
    exner_top = 1.0 - G * ztop / (CP_D * theta0)
    p_top = P0 * exner_top ** (CP_D / R_D)
    eta = np.linspace(1.0, 0.0, nz + 1)
    m = flat_metrics(eta, ny, nx, p_top)
    ht = _spectral_terrain(ny, nx, hmax, seed)
    psb = P0 * (1.0 - G * ht / (CP_D * theta0)) ** (CP_D / R_D)
    mub = psb - p_top
    eta_mass = 0.5 * (eta[:-1] + eta[1:])
    pb = eta_mass[:, None, None] * mub[None] + p_top
    z = CP_D * theta0 / G * (1.0 - (pb / P0) ** (R_D / CP_D))
    theta = theta_s * np.exp(nbv ** 2 * z / G)
    zfrac = np.clip(z / ztop, 0.0, 1.0)
    ubar = 5.0 + 15.0 * zfrac
    u = np.zeros((nz, ny, nx + 1))
    v = np.zeros((nz, ny + 1, nx))
    u[:, :, :nx] = ubar + 0.5 * rng.standard_normal((nz, ny, nx))
    u[:, :, nx] = u[:, :, 0]
    v[:, :ny, :] = 0.5 * rng.standard_normal((nz, ny, nx))
    v[:, ny, :] = v[:, 0, :]
    t = theta * (pb / P0) ** (R_D / CP_D)
    qv = 0.8 * _qsat(t, pb) * np.exp(-z / 8000.0)
    band = ((z >= 2000.0) & (z <= 6000.0)).astype(np.float64)
    qc = band * np.exp(rng.normal(np.log(1.0e-4), 0.5, size=z.shape))
    qr = band * np.exp(rng.normal(np.log(5.0e-5), 0.5, size=z.shape))
    moist = dict(qv=qv, qc=qc, qr=qr, qi=np.zeros_like(qv), qs=np.zeros_like(qv), qg=np.zeros_like(qv))
    s = _balanced_state(m, theta, np.full_like(theta, theta0), mub, ht, u, v, moist)
    c = _controls(dt_s=dt, acoustic_substeps=ns, epssm=0.1, top_lid=False, moist_adv_opt=1,
                  run_boundary=specified, bc_ideal=not specified)
    if specified:
        brng = np.random.default_rng(seed + 101) if bdy_noise else None
        for k, val in _boundary_leaves(s, nz, ny, nx, rng=brng).items():
            setattr(s, k, val)
    return Case("real_like_moist", nx, ny, nz, m, dict(c, dx=dx, dy=dx), s, np.zeros((ny, nx)),
                notes={"seed": seed, "hmax": hmax})


def mountain_wave(nx: int = 256, ny: int = 256, nz: int = 50, *, dx: float = 2000.0, ztop: float = 25000.0,
                  dt: float = 12.0, ns: int = 6) -> Case:
    """3-D mountain wave: Witch-of-Agnesi hill (1 km high, 10 km half-width), constant
    N = 0.01 from theta_s = 288 K, uniform u = 10 m/s, stretched eta
    ``eta_k = 1 - (exp(2 s_k) - 1)/(e^2 - 1)`` with ``s_k = k/nz`` (finer near the
    ground), Rayleigh damping (damp_opt 3, dampcoef 0.2) in the top 5 km, specified
    boundaries with constant strips, dt 12 s, 6 substeps."""
    theta0 = 300.0
    exner_top = 1.0 - G * ztop / (CP_D * theta0)
    p_top = P0 * exner_top ** (CP_D / R_D)
    sk = np.arange(nz + 1) / nz
    eta = 1.0 - (np.exp(2.0 * sk) - 1.0) / (np.exp(2.0) - 1.0)
    m = flat_metrics(eta, ny, nx, p_top)
    x = (np.arange(nx) + 0.5 - 0.5 * nx) * dx
    y = (np.arange(ny) + 0.5 - 0.5 * ny) * dx
    rr2 = x[None, :] ** 2 + y[:, None] ** 2
    ht = 1000.0 / (1.0 + rr2 / 10000.0 ** 2) ** 1.5
    psb = P0 * (1.0 - G * ht / (CP_D * theta0)) ** (CP_D / R_D)
    mub = psb - p_top
    eta_mass = 0.5 * (eta[:-1] + eta[1:])
    pb = eta_mass[:, None, None] * mub[None] + p_top
    z = CP_D * theta0 / G * (1.0 - (pb / P0) ** (R_D / CP_D))
    theta = 288.0 * np.exp(0.01 ** 2 * z / G)
    u = np.full((nz, ny, nx + 1), 10.0)
    v = np.zeros((nz, ny + 1, nx))
    s = _balanced_state(m, theta, np.full_like(theta, theta0), mub, ht, u, v)
    c = _controls(dt_s=dt, acoustic_substeps=ns, epssm=0.1, top_lid=False, damp_opt=3, dampcoef=0.2,
                  zdamp=5000.0, run_boundary=True, bc_ideal=False)
    for k, val in _boundary_leaves(s, nz, ny, nx).items():
        setattr(s, k, val)
    return Case("mountain_wave", nx, ny, nz, m, dict(c, dx=dx, dy=dx), s, np.zeros((ny, nx)))


def crop(case: Case, nx: int, ny: int, j0: int = 0, i0: int = 0, *, full_leaves: bool = False) -> Case:
    """Sub-window ``[j0:j0+ny, i0:i0+nx]`` of a case (periodic wrap of the
    staggered edge faces), for parity runs on windows of a full-size case.  A
    case with boundary strips gets constant strips rebuilt from the window's
    edge rows (``full_leaves``: also the strips of the end-of-step boundary
    pass)."""
    s = case.state
    m = case.metrics
    n = SimpleNamespace()
    jy, ix = slice(j0, j0 + ny), slice(i0, i0 + nx)
    if j0 + ny > case.ny or i0 + nx > case.nx or j0 < 0 or i0 < 0:
        raise ValueError("crop window outside the case")
    for k, vv in vars(s).items():
        if k.endswith("_bdy"):
            continue
        if k == "u":
            a = vv[:, jy, i0:i0 + nx + 1].copy()
            a[:, :, nx] = a[:, :, 0]
        elif k == "v":
            a = vv[:, j0:j0 + ny + 1, ix].copy()
            a[:, ny, :] = a[:, 0, :]
        elif vv.ndim == 3:
            a = vv[:, jy, ix].copy()
        else:
            a = vv[jy, ix].copy()
        setattr(n, k, a)
    mm = SimpleNamespace(**vars(m))
    for k in ("msftx", "msfty", "f", "e", "sina", "cosa"):
        setattr(mm, k, getattr(m, k)[jy, ix].copy())
    for k in ("msfux", "msfuy"):
        setattr(mm, k, getattr(m, k)[jy, i0:i0 + nx + 1].copy())
    for k in ("msfvx", "msfvy"):
        setattr(mm, k, getattr(m, k)[j0:j0 + ny + 1, ix].copy())
    if hasattr(s, "u_bdy") or full_leaves:
        for kk, val in _boundary_leaves(n, case.nz, ny, nx, full=full_leaves).items():
            setattr(n, kk, val)
    return Case(case.name + f"_crop{nx}x{ny}", nx, ny, case.nz, mm, dict(case.controls), n,
                case.mudf[jy, ix].copy(), notes=dict(case.notes, crop=(j0, i0)))


def with_full_leaves(case: Case, rng=None) -> Case:
    """The case with every boundary strip the end-of-step lateral boundary
    pass reads, built from its initial edge rows (``rng``: the dynamic strips
    perturbed and drifting in time as ``_boundary_leaves`` does)."""
    for kk, val in _boundary_leaves(case.state, case.nz, case.ny, case.nx, rng=rng, full=True).items():
        setattr(case.state, kk, val)
    return case
