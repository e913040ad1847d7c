"""The oracle's nest coupling pinned to the reference's known answers
(tests/test_p0_1a_nesting.py, tests/test_v0110_boundary_feedback.py,
tests/test_v0120_feedback_smoother.py): the sint registration reproduces a
linear parent field exactly and sits -(ratio//2)/ratio of a parent cell from
the node-aligned one; the ring strips run outer to inner; the boundary
package is a two-time leaf of the child's ring and the parent's; the mass
feedback is the child mean over each parent cell and conserves the overlap
integral; U / V feedback average ratio donors along the other axis; sm121
equals WRF's index loops, leaves the outside untouched and keeps a constant
field; the state feedback rebuilds totals from the parent base."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle import nesting as N

RATIO, IPOS, JPOS = 3, 4, 3
PNX, PNY = 20, 16
CNX, CNY = 27, 24


def _w(**kw):
    c = dict(ratio=RATIO, i_parent_start=IPOS, j_parent_start=JPOS, parent_ny=PNY, parent_nx=PNX, child_ny=CNY,
             child_nx=CNX)
    c.update(kw)
    return N.build_interp_weights(**c)


def test_sint_reproduces_a_linear_field_exactly():
    w = _w()
    jj, ii = np.meshgrid(np.arange(PNY, dtype=float), np.arange(PNX, dtype=float), indexing="ij")
    f = (2.5 + 0.75 * ii - 1.25 * jj)[None]
    got = N.interp(f, w)
    x = (IPOS - 1) + (np.arange(CNX) - RATIO // 2) / RATIO
    y = (JPOS - 1) + (np.arange(CNY) - RATIO // 2) / RATIO
    want = 2.5 + 0.75 * np.clip(x, 0, PNX - 1)[None, :] - 1.25 * np.clip(y, 0, PNY - 1)[:, None]
    np.testing.assert_allclose(got[0], want, rtol=0, atol=1e-12)


def test_sint_registration_offset_from_the_node_aligned_one():
    s, b = _w(registration="sint"), _w(registration="bilinear")
    xs = s.x0 + s.wx
    xb = b.x0 + b.wx
    inner = (xs > 0) & (xb < PNX - 1)
    np.testing.assert_allclose((xb - xs)[inner], (RATIO // 2) / RATIO, atol=1e-12)


def test_ring_strips_run_outer_to_inner():
    z, ny, nx, w = 2, 7, 9, 3
    f = np.arange(z * ny * nx, dtype=float).reshape(z, ny, nx)
    s = N.field_sides_3d(f, w, 12)
    assert s.shape == (4, w, z, 12)
    np.testing.assert_array_equal(s[0, 1, :, :ny], f[:, :, 1])           # W: column 1
    np.testing.assert_array_equal(s[1, 0, :, :ny], f[:, :, nx - 1])      # E: the east column first
    np.testing.assert_array_equal(s[2, 2, :, :nx], f[:, 2, :])           # S: row 2
    np.testing.assert_array_equal(s[3, 0, :, :nx], f[:, ny - 1, :])      # N: the north row first
    assert np.all(s[0, :, :, ny:] == 0.0) and np.all(s[2, :, :, nx:] == 0.0)


def nest_pair(seed=0, nz=6):
    rng = np.random.default_rng(seed)
    side = max(CNX, CNY) + 1

    def state(ny, nx, bdy):
        s = SimpleNamespace(u=rng.standard_normal((nz, ny, nx + 1)), v=rng.standard_normal((nz, ny + 1, nx)),
                            w=rng.standard_normal((nz + 1, ny, nx)), theta=300.0 + rng.standard_normal((nz, ny, nx)),
                            qv=1e-3 * rng.random((nz, ny, nx)), qc=1e-4 * rng.random((nz, ny, nx)),
                            qr=1e-4 * rng.random((nz, ny, nx)), qi=np.zeros((nz, ny, nx)),
                            qs=np.zeros((nz, ny, nx)), qg=np.zeros((nz, ny, nx)),
                            p_perturbation=50.0 * rng.standard_normal((nz, ny, nx)),
                            ph_perturbation=20.0 * rng.standard_normal((nz + 1, ny, nx)),
                            mu_perturbation=30.0 * rng.standard_normal((ny, nx)))
        s.p_total = 5.0e4 + 100.0 * rng.random((nz, ny, nx)) + s.p_perturbation
        s.ph_total = 2.0e4 + 10.0 * rng.random((nz + 1, ny, nx)) + s.ph_perturbation
        s.mu_total = 9.0e4 + 50.0 * rng.random((ny, nx)) + s.mu_perturbation
        if bdy:
            for name, lev in (("u_bdy", nz), ("v_bdy", nz), ("w_bdy", nz + 1), ("theta_bdy", nz), ("qv_bdy", nz),
                              ("ph_bdy", nz + 1), ("phb_bdy", nz + 1), ("p_bdy", nz), ("pb_bdy", nz),
                              ("mu_bdy", 1), ("mub_bdy", 1)):
                setattr(s, name, rng.standard_normal((2, 4, 5, lev, side)))
        return s

    return state(CNY, CNX, True), state(PNY, PNX, False)


def test_boundary_package_is_a_two_time_leaf_of_child_and_parent_rings():
    child, parent = nest_pair()
    wts = N.build_nest_force_weights(ratio=RATIO, i_parent_start=IPOS, j_parent_start=JPOS, parent_ny=PNY,
                                     parent_nx=PNX, child_ny=CNY, child_nx=CNX)
    out = N.build_child_boundary_package(child, parent, wts)
    side = out.u_bdy.shape[-1]
    np.testing.assert_array_equal(out.theta_bdy[0], N.field_sides_3d(child.theta, 5, side))
    np.testing.assert_array_equal(out.theta_bdy[1], N.field_sides_3d(N.interp(parent.theta, wts.mass), 5, side))
    np.testing.assert_array_equal(out.u_bdy[1], N.field_sides_3d(N.interp(parent.u, wts.u), 5, side))
    phb = child.ph_total - child.ph_perturbation
    np.testing.assert_array_equal(out.phb_bdy[0], out.phb_bdy[1])
    np.testing.assert_array_equal(out.phb_bdy[0], N.field_sides_3d(phb, 5, side))
    assert out.mu_bdy.shape == (2, 4, 5, 1, side)
    np.testing.assert_array_equal(out.qv, child.qv)  # the interior is untouched


def _plans(**kw):
    c = dict(ratio=RATIO, i_parent_start=IPOS, j_parent_start=JPOS, parent_nx=PNX, parent_ny=PNY, child_nx=CNX,
             child_ny=CNY)
    c.update(kw)
    return N.build_state_feedback_plans(**c)


def test_mass_feedback_is_the_child_cell_mean_and_conserves_the_overlap():
    child, parent = nest_pair(1)
    p = _plans().mass
    fed = N.apply_feedback(parent.theta, child.theta, p)
    for n in (0, len(p.parent_lin) // 2, len(p.parent_lin) - 1):
        pj, pi = divmod(int(p.parent_lin[n]), p.pwe)
        cj0 = (pj + 1 - JPOS) * RATIO  # child rows of parent row pj + 1 (1-based)
        ci0 = (pi + 1 - IPOS) * RATIO
        want = child.theta[:, cj0:cj0 + RATIO, ci0:ci0 + RATIO].mean(axis=(1, 2))
        np.testing.assert_allclose(fed[:, pj, pi], want, rtol=1e-14)
    donors = np.unique(p.child_lin.ravel())
    flat_c = child.theta.reshape(child.theta.shape[0], -1)
    flat_f = fed.reshape(fed.shape[0], -1)
    np.testing.assert_allclose(flat_f[:, p.parent_lin].sum(axis=1) * RATIO ** 2, flat_c[:, donors].sum(axis=1),
                               rtol=1e-13)
    out_mask = np.ones(PNY * PNX, bool)
    out_mask[p.parent_lin] = False
    np.testing.assert_array_equal(flat_f[:, out_mask], parent.theta.reshape(parent.theta.shape[0], -1)[:, out_mask])


def test_staggered_feedback_stencils():
    pl = _plans()
    assert pl.u.stencil == RATIO and pl.v.stencil == RATIO and pl.mass.stencil == RATIO ** 2
    for n in range(len(pl.u.parent_lin)):
        rows, cols = np.divmod(pl.u.child_lin[n], pl.u.cwe)
        assert len(set(cols)) == 1 and np.all(np.diff(rows) == 1)  # one u column, consecutive rows
        rows, cols = np.divmod(pl.v.child_lin[n if n < len(pl.v.parent_lin) else 0], pl.v.cwe)
        assert len(set(rows)) == 1 and np.all(np.diff(cols) == 1)


def _sm121_wrf_loops(f, i_lo_1, i_hi_1, j_lo_1, j_hi_1):
    """WRF sm121's serial loops (1-based inclusive bounds): j pass, i pass."""
    cf, cnew = f.copy(), f.copy()
    for i1 in range(i_lo_1, i_hi_1 + 1):
        for j1 in range(j_lo_1, j_hi_1 + 1):
            i, j = i1 - 1, j1 - 1
            cnew[j, i] = 0.25 * (cf[j + 1, i] + 2.0 * cf[j, i] + cf[j - 1, i])
    for j1 in range(j_lo_1, j_hi_1 + 1):
        for i1 in range(i_lo_1, i_hi_1 + 1):
            i, j = i1 - 1, j1 - 1
            cf[j, i] = 0.25 * (cnew[j, i + 1] + 2.0 * cnew[j, i] + cnew[j, i - 1])
    return cf


def test_sm121_equals_the_wrf_loops_per_stagger():
    rng = np.random.default_rng(3)
    pl = _plans()
    for stag, sm, shape in (("", pl.mass_smooth, (PNY, PNX)), ("U", pl.u_smooth, (PNY, PNX + 1)),
                            ("V", pl.v_smooth, (PNY + 1, PNX))):
        f = rng.standard_normal(shape)
        istag, jstag = (0 if stag == "U" else 1), (0 if stag == "V" else 1)
        want = _sm121_wrf_loops(f, IPOS + 2, IPOS + CNX // RATIO - 2 - istag, JPOS + 2,
                                JPOS + CNY // RATIO - 2 - jstag)
        np.testing.assert_array_equal(N.sm121(f, sm), want)
    c = np.full((PNY, PNX), 7.0)
    np.testing.assert_array_equal(N.sm121(c, pl.mass_smooth), c)


def test_state_feedback_rebuilds_totals_from_the_parent_base():
    child, parent = nest_pair(2)
    out = N.apply_state_feedback(parent, child, _plans())
    np.testing.assert_allclose(out.p_total - out.p_perturbation, parent.p_total - parent.p_perturbation, rtol=1e-15)
    np.testing.assert_allclose(out.mu_total - out.mu_perturbation, parent.mu_total - parent.mu_perturbation,
                               rtol=1e-15)
    assert not np.array_equal(out.theta, parent.theta)
    same = N.apply_state_feedback(parent, child, _plans(), feedback=False)
    assert same is parent
