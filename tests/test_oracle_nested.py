"""Oracle pins: the nested child boundary (``force_geopotential=False``).

A nested child runs the specified domain's non-periodic step with the
specified-only advection degradation and boundary cadence off, plus three
opt-in in-loop forcings (operational_mode.py:1906-1968): the relax-zone ph'
and w tendencies (coupling/boundary_apply.py:1045-1087) and the ring-0 ph'
pin after advance_w (boundary_apply.py:1299-1340).  Pinned here: the relax
tendency against a literal per-cell restatement of WRF's relax_bdytend
stencil, the ring-0 ph' of a finished step against the ph' leaf at the
step's lead, and the nested step without forcings against the plain
specified step.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import dycore as D
from tests import parity_util as P
from tests.test_oracle_bdy_cadence import _relax_literal
from wrf_gpu_b200 import cases


def test_nested_relax_matches_the_literal_stencil():
    rng = np.random.default_rng(424242)
    nzp, ny, nx, dt = 4, 13, 15, 12.0
    field = 5.0 * rng.normal(size=(nzp, ny, nx))
    target = 5.0 * rng.normal(size=(nzp, ny, nx))
    mut = 950.0 + rng.normal(size=(ny, nx))
    m = SimpleNamespace(c1f=0.9 + 0.02 * np.arange(nzp), c2f=40.0 + np.arange(nzp),
                        msfty=1.0 + 0.001 * rng.normal(size=(ny, nx)))
    got = D.nested_relax_tendency(field, target, mut, m, dt)
    mass_f = m.c1f[:, None, None] * mut[None] + m.c2f[:, None, None]
    want = _relax_literal(mass_f * field, mass_f * target, dt) / m.msfty[None]
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
    # only the relax rows 1..3 carry a tendency
    assert np.all(got[:, 0, :] == 0.0) and np.all(got[:, :, 0] == 0.0)
    assert np.all(got[:, 4:-4, 4:-4] == 0.0)


def _nested_case(**controls):
    case = cases.real_like_moist(24, 20, 10, hmax=600.0, specified=True, bdy_noise=True)
    case.controls.update(force_geopotential=False, **controls)
    return case


def test_nested_without_forcings_is_the_plain_specified_step():
    # the degradation and cadence flags are specified-only: a nested child ignores them
    nested = P.oracle_steps(_nested_case(specified_adv_degrade=True, specified_bdy_cadence=True), 1, lead0=600.0)
    plain = P.oracle_steps(cases.real_like_moist(24, 20, 10, hmax=600.0, specified=True, bdy_noise=True), 1,
                           lead0=600.0)
    for k in P.STATE_KEYS:
        np.testing.assert_array_equal(getattr(nested.state, k), getattr(plain.state, k), err_msg=k)


def test_nested_ph_spec_pins_ring0_ph_to_the_leaf_at_the_lead():
    lead = 1800.0
    case = _nested_case(nested_ph_spec=True)
    out = P.oracle_steps(case, 1, lead0=lead)
    s = out.state
    nz = s.theta.shape[0]
    ny, nx = s.mu_total.shape
    leaf = D.interpolate_boundary_leaf(case.state.ph_bdy, lead, case.controls["update_cadence_s"])
    ring = D.full_ring_target(leaf, nz + 1, ny, nx)
    php = s.ph_perturbation
    for sl in ((slice(None), 0, slice(None)), (slice(None), ny - 1, slice(None)),
               (slice(None), slice(None), 0), (slice(None), slice(None), nx - 1)):
        np.testing.assert_allclose(php[sl], ring[sl], rtol=1e-12, atol=1e-9)
    free = P.oracle_steps(_nested_case(), 1, lead0=lead).state.ph_perturbation
    assert np.abs(free[:, 0, :] - ring[:, 0, :]).max() > 1e-3


def test_nested_relax_forcings_change_the_step():
    base = P.oracle_steps(_nested_case(), 1, lead0=600.0).state
    for kw in (dict(nested_ph_relax=True), dict(nested_w_relax=True)):
        s = P.oracle_steps(_nested_case(**kw), 1, lead0=600.0).state
        for k in ("u", "v", "w", "theta", "ph_perturbation", "mu_perturbation"):
            assert np.isfinite(getattr(s, k)).all(), (kw, k)
        assert np.abs(s.ph_perturbation - base.ph_perturbation).max() > 1e-6, kw
