"""Multi-GPU form of the RK3 step: a y-slab decomposition with wide halos.

The reference shards its forecast into x slabs whose periodic halos are
refreshed by ``lax.ppermute`` inside the operators
(``runtime/sharding.py:260-415, 800-866``; specified boundaries are rejected
there, ``:286-290``).  Here each rank owns a band of rows of the (nz, ny, nx)
arrays -- a band of rows is contiguous on every level, so a halo block is nz
contiguous runs -- and steps its band plus ``H`` halo rows on each side with
the unchanged single-domain step.  Rows that the local step gets wrong (the
slab's own edges, treated as domain edges) lie in the halos; after each step
the ranks exchange the halo blocks of the fields the next step reads, one
packed message per neighbour and direction (``wrfgpu_rows_pack`` /
``wrfgpu_rows_unpack``; NCCL point-to-point between ranks, or a plain
buffer hand-over when one process drives every slab).  One exchange per RK3
step instead of one per acoustic substep: the halo is wide enough to cover
how far one whole step carries information (``halo_rows``).

The reference's operators roll their neighbours around the domain even under
specified boundaries (the flux-form advection, the positive-definite
limiter, the 6th-order and Smagorinsky filters), so the rows next to the
south edge read the rows next to the north edge within the same stage.  The
first and last slabs therefore carry the rows across the domain edge as their
far-side halo, placed so that the domain's row 0 is the slab's first row and
its row ny-1 the slab's last: the first slab holds rows
``[0, own_hi + H) ++ [ny - H, ny)``, the last ``[0, H) ++ [own_lo - H, ny)``.
Every slab then sees the domain edges exactly where the whole-domain step
sees them, the halo exchange is a ring, and the owned rows match the
whole-domain step bit for bit (periodic and specified domains alike).

Not sharded: constant-K diffusion (its mean layer depth is a domain-wide
mean) and the post-step guards (domain sums); the end-of-step lateral
boundary pass is (``boundary_pass=True``).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, replace

import numpy as np
import torch

from . import _capi, dycore

EXCHANGED_STATE = ("u", "v", "w", "theta", "p_total", "p_perturbation", "ph_total", "ph_perturbation", "mu_total",
                   "mu_perturbation") + dycore.MOIST
EXCHANGED_CARRY = ("mudf",)
_ROW_METRICS = ("msftx", "msfty", "msfux", "msfuy", "f", "e", "sina", "cosa")
_FACE_METRICS = ("msfvx", "msfvy")


def halo_rows(nl: dycore.OperationalNamelist) -> int:
    """Halo rows per side for one exchange per RK3 step.

    One step carries information ``1 + ns/2 + ns`` rows through the acoustic
    substeps of its three stages (one row per substep) and a few rows per
    stage through the large-step stencils (5th-order fluxes, the limiter, the
    filters): ``10 + ns + ceil(ns/2)`` covers it with margin (measured on the
    oracle: 11, 16 and 20 rows for ns = 2, 6 and 10 with both filters and the
    boundary cadence).  A slab's own edge is treated as a domain edge, which
    spoils its boundary zone (spec_zone + relax_zone rows) before the step
    starts; those rows are added under specified boundaries."""
    if nl.const_nu_m2_s > 0.0:
        raise NotImplementedError("constant-K diffusion reads a domain-wide mean layer depth; it is not sharded")
    ns = max(1, int(nl.acoustic_substeps))
    h = 10 + ns + (ns + 1) // 2
    if nl.run_boundary and nl.bc_source != "ideal":
        h += int(nl.boundary_config.spec_zone) + int(nl.boundary_config.relax_zone)
    return h


@dataclass(frozen=True)
class SlabLayout:
    """Rank ``rank``'s slab of a ``world``-way split of ``ny`` rows.

    ``rows[l]`` is the global row of local row ``l``; ``own_local``,
    ``below_local`` and ``above_local`` are the local rows where the owned
    band, the block from the rank below (global rows ``own_lo - H ..
    own_lo``, modulo ny) and the block from the rank above (``own_hi ..
    own_hi + H``) start."""

    ny: int
    world: int
    rank: int
    halo: int
    own_lo: int
    own_hi: int
    rows: tuple
    own_local: int
    below_local: int
    above_local: int

    @property
    def n_local(self) -> int:
        return len(self.rows)

    @property
    def own(self) -> int:
        return self.own_hi - self.own_lo

    def faces(self) -> np.ndarray:
        """Global y-face of each local y-face: the south face of every local
        row, then the north face of the last one."""
        r = np.asarray(self.rows)
        return np.concatenate([r, [r[-1] + 1]])

    @property
    def below(self) -> int:
        return (self.rank - 1) % self.world

    @property
    def above(self) -> int:
        return (self.rank + 1) % self.world


def own_bounds(ny: int, world: int, rank: int) -> tuple[int, int]:
    return rank * ny // world, (rank + 1) * ny // world


def slab_layout(ny: int, world: int, rank: int, halo: int) -> SlabLayout:
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the decomposition")
    lo, hi = own_bounds(ny, world, rank)
    if world == 1:
        return SlabLayout(ny, 1, 0, 0, 0, ny, tuple(range(ny)), 0, 0, 0)
    if ny // world < halo:
        raise ValueError(f"{world} slabs of {ny} rows own fewer rows than the {halo}-row halo; use fewer ranks")
    own = hi - lo
    window = [(lo - halo + t) % ny for t in range(own + 2 * halo)]
    pos = {"below": 0, "own": halo, "above": halo + own}
    k = 0
    for t in range(1, len(window)):
        if window[t] == 0 and window[t - 1] == ny - 1:
            k = t  # the domain edge inside the window: rotate it to the slab's start
    n = len(window)
    rows = tuple(window[k:] + window[:k])
    loc = {name: (p - k) % n for name, p in pos.items()}
    return SlabLayout(ny, world, rank, halo, lo, hi, rows, loc["own"], loc["below"], loc["above"])


def _runs(src_rows: np.ndarray):
    """(dst_start, src_start, length) runs of consecutive source rows."""
    out, start = [], 0
    for t in range(1, len(src_rows) + 1):
        if t == len(src_rows) or src_rows[t] != src_rows[t - 1] + 1:
            out.append((start, int(src_rows[start]), t - start))
            start = t
    return out


def _as3(t: torch.Tensor) -> torch.Tensor:
    return t if t.dim() == 3 else t.unsqueeze(0)


class CudaRows:
    """Row movement on the device through ``libwrfgpu.so``."""

    def __init__(self):
        self.lib = _capi.load()

    def copy(self, src, src_row0, dst, dst_row0, nrows, stream=None):
        s3, d3 = _as3(src), _as3(dst)
        for t in (s3, d3):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("row copies take contiguous float64 CUDA tensors")
        if s3.shape[0] != d3.shape[0] or s3.shape[2] != d3.shape[2]:
            raise ValueError("row copies need the same levels and row length on both sides")
        st = torch.cuda.current_stream(src.device) if stream is None else stream
        nz, sny, nx = s3.shape
        _capi.check(self.lib.wrfgpu_copy_rows(ctypes.c_void_p(s3.data_ptr()), nz, sny, int(src_row0),
                                              ctypes.c_void_p(d3.data_ptr()), d3.shape[1], int(dst_row0),
                                              int(nrows), nx, ctypes.c_void_p(st.cuda_stream)))

    def _blocks(self, blocks):
        if len(blocks) > _capi.MAX_ROW_BLOCKS:
            raise ValueError("too many row blocks for one launch")
        arr = (_capi.RowBlock * max(1, len(blocks)))()
        for k, (t, row0, nrows, offset) in enumerate(blocks):
            t3 = _as3(t)
            if not (t3.is_cuda and t3.dtype == torch.float64 and t3.is_contiguous()):
                raise ValueError("row blocks take contiguous float64 CUDA tensors")
            nz, ny, nx = t3.shape
            arr[k] = _capi.RowBlock(t3.data_ptr(), nz, ny, nx, int(row0), int(nrows), int(offset))
        return arr

    def pack(self, blocks, buffer, stream=None):
        st = torch.cuda.current_stream(buffer.device) if stream is None else stream
        _capi.check(self.lib.wrfgpu_rows_pack(self._blocks(blocks), len(blocks), ctypes.c_void_p(buffer.data_ptr()),
                                              buffer.numel(), ctypes.c_void_p(st.cuda_stream)))

    def unpack(self, blocks, buffer, stream=None):
        st = torch.cuda.current_stream(buffer.device) if stream is None else stream
        _capi.check(self.lib.wrfgpu_rows_unpack(self._blocks(blocks), len(blocks),
                                                ctypes.c_void_p(buffer.data_ptr()), buffer.numel(),
                                                ctypes.c_void_p(st.cuda_stream)))


def take_rows(copier, src: torch.Tensor, rows: np.ndarray) -> torch.Tensor:
    """A new array of ``src``'s rows ``rows`` (axis -2), in that order."""
    shape = list(src.shape)
    shape[-2] = len(rows)
    out = torch.empty(shape, dtype=src.dtype, device=src.device)
    for d0, s0, n in _runs(np.asarray(rows)):
        copier.copy(src, s0, out, d0, n)
    return out


def _slice_leaf(leaf: torch.Tensor, rows: np.ndarray, faces: np.ndarray, is_v: bool, nx: int) -> torch.Tensor:
    """A boundary strip (ntime, 4, width, z, side_len) for the slab: the W / E
    strips (indexed by row, by face for v) gathered at the slab's rows, the
    S / N strips unchanged."""
    q = faces if is_v else rows
    nt, _, width, lz, side = leaf.shape
    side_l = max(side, nx + 1, len(faces))
    out = torch.zeros((nt, 4, width, lz, side_l), dtype=leaf.dtype, device=leaf.device)
    idx = torch.as_tensor(np.asarray(q), dtype=torch.long, device=leaf.device)
    out[:, :2, ..., :len(q)] = leaf[:, :2].index_select(-1, idx)
    out[:, 2:, ..., :side] = leaf[:, 2:]
    return out


def slab_namelist(nl: dycore.OperationalNamelist, layout: SlabLayout, copier) -> dycore.OperationalNamelist:
    """The namelist of one slab: ny, the 2-D metrics and the base tendencies
    taken at the slab's rows (y-face arrays at its faces)."""
    rows, faces = np.asarray(layout.rows), layout.faces()
    m = nl.metrics
    kw = {n: take_rows(copier, getattr(m, n), rows) for n in _ROW_METRICS}
    kw.update({n: take_rows(copier, getattr(m, n), faces) for n in _FACE_METRICS})
    t = nl.tendencies
    tend = dycore.Tendencies(**{n: (None if getattr(t, n) is None else
                                    take_rows(copier, getattr(t, n), faces if n == "v" else rows))
                                for n in ("u", "v", "w", "theta", "mu")})
    return replace(nl, ny=layout.n_local, metrics=replace(m, **kw), tendencies=tend)


def slab_state(state: dycore.State, layout: SlabLayout, copier, nx: int) -> dycore.State:
    rows, faces = np.asarray(layout.rows), layout.faces()
    kw = {}
    for name in dycore.State.__dataclass_fields__:
        t = getattr(state, name)
        if t is None:
            kw[name] = None
        elif name.endswith("_bdy"):
            kw[name] = _slice_leaf(t, rows, faces, name == "v_bdy", nx)
        else:
            kw[name] = take_rows(copier, t, faces if name == "v" else rows)
    return dycore.State(**kw)


class SlabStepper:
    """One rank's slab: its namelist, carry and halo blocks.

    ``step_fn(carry, namelist, lead_seconds) -> carry`` advances a slab
    (default: ``dycore.rk_scan_step``, then with ``boundary_pass`` the
    end-of-step lateral boundary pass); ``copier`` moves rows (default: the
    CUDA kernels)."""

    def __init__(self, nl: dycore.OperationalNamelist, layout: SlabLayout, *, boundary_pass: bool = False,
                 copier=None, step_fn=None):
        self.layout = layout
        self.global_nl = nl
        self.copier = CudaRows() if copier is None else copier
        self.nl = slab_namelist(nl, layout, self.copier)
        self.boundary_pass = bool(boundary_pass)
        self.step_fn = self._default_step if step_fn is None else step_fn
        self.carry = None

    def _default_step(self, carry, nl, lead_seconds):
        nxt = dycore.rk_scan_step(carry, nl, lead_seconds=lead_seconds)
        if self.boundary_pass and nl.run_boundary:
            state, _ = dycore.step_epilogue(nxt.state, carry.state, lead_seconds, replace(nl, disable_guards=True))
            nxt = nxt.replace(state=state)
        return nxt

    def load(self, carry: dycore.OperationalCarry) -> None:
        """Take this slab's rows of a whole-domain carry (state, strips, mudf)."""
        st = slab_state(carry.state, self.layout, self.copier, self.global_nl.nx)
        mudf = carry.mudf if carry.mudf is not None else torch.zeros_like(carry.state.mu_total)
        self.carry = dycore.initial_operational_carry(st).replace(
            mudf=take_rows(self.copier, mudf, np.asarray(self.layout.rows)))

    def advance(self, lead_seconds) -> None:
        self.carry = self.step_fn(self.carry, self.nl, lead_seconds)

    # ---- halo blocks ------------------------------------------------------
    def _fields(self):
        c = self.carry
        out = [(n, getattr(c.state, n)) for n in EXCHANGED_STATE if getattr(c.state, n) is not None]
        return out + [(n, getattr(c, n)) for n in EXCHANGED_CARRY]

    def _blocks(self, start_local: int, first_global: int):
        """Row blocks of every exchanged field for H rows from local row
        ``start_local`` whose first global row is ``first_global``; a v
        block that ends at the domain's last row also carries its north face."""
        H, ny = self.layout.halo, self.layout.ny
        ends_at_top = (first_global + H - 1) % ny == ny - 1
        blocks, off = [], 0
        for name, t in self._fields():
            t3 = _as3(t)
            n = H + 1 if (name == "v" and ends_at_top) else H
            blocks.append((t, start_local, n, off))
            off += t3.shape[0] * n * t3.shape[2]
        return blocks, off

    def send_blocks(self):
        """(to the rank below, to the rank above): this slab's first and last
        H owned rows."""
        L = self.layout
        down = self._blocks(L.own_local, L.own_lo)
        up = self._blocks(L.own_local + L.own - L.halo, L.own_hi - L.halo)
        return down, up

    def recv_blocks(self):
        """(from the rank below, from the rank above)."""
        L = self.layout
        below = self._blocks(L.below_local, (L.own_lo - L.halo) % L.ny)
        above = self._blocks(L.above_local, L.own_hi % L.ny)
        return below, above

    def pack(self):
        (down, nd), (up, nu) = self.send_blocks()
        dev = self.carry.state.theta.device
        bd = torch.empty(nd, dtype=torch.float64, device=dev)
        bu = torch.empty(nu, dtype=torch.float64, device=dev)
        self.copier.pack(down, bd)
        self.copier.pack(up, bu)
        return bd, bu

    def unpack(self, from_below: torch.Tensor, from_above: torch.Tensor) -> None:
        (below, _), (above, _) = self.recv_blocks()
        self.copier.unpack(below, from_below)
        self.copier.unpack(above, from_above)

    def recv_sizes(self) -> tuple[int, int]:
        (_, nb), (_, na) = self.recv_blocks()
        return nb, na

    # ---- owned rows -------------------------------------------------------
    def owned_into(self, out: dycore.OperationalCarry, state_names=None, carry_names=None) -> None:
        """Copy this slab's owned rows into a whole-domain carry ``out``."""
        L = self.layout
        top = L.own_hi == L.ny
        pairs = []
        for n in (state_names or [f for f in dycore.State.__dataclass_fields__ if not f.endswith("_bdy")]):
            pairs.append((n, getattr(self.carry.state, n), getattr(out.state, n)))
        for n in (carry_names or ("mudf", "t_2ave", "ww", "muave", "muts", "ph_tend", "u_save", "v_save", "w_save",
                                  "t_save", "ph_save", "mu_save", "ww_save")):
            pairs.append((n, getattr(self.carry, n), getattr(out, n)))
        for n, src, dst in pairs:
            if src is None or dst is None:
                continue
            extra = 1 if (n in ("v", "v_save") and top) else 0
            self.copier.copy(src, L.own_local, dst, L.own_lo, L.own + extra)


def _like_global(carry: dycore.OperationalCarry) -> dycore.OperationalCarry:
    e = lambda t: None if t is None else torch.empty_like(t)
    st = dycore.State(**{n: (getattr(carry.state, n) if n.endswith("_bdy") else e(getattr(carry.state, n)))
                         for n in dycore.State.__dataclass_fields__})
    s = carry.state
    return dycore.OperationalCarry(state=st, t_2ave=e(s.theta), ww=e(s.w), mudf=e(s.mu_total), muave=e(s.mu_total),
                                   muts=e(s.mu_total), ph_tend=e(s.w), u_save=e(s.u), v_save=e(s.v), w_save=e(s.w),
                                   t_save=e(s.theta), ph_save=e(s.w), mu_save=e(s.mu_total), ww_save=e(s.w))


class SlabRing:
    """Every slab of a decomposition driven from one process (one device or
    several): each step advances every slab, then hands each slab's packed
    send blocks to its neighbours."""

    def __init__(self, nl: dycore.OperationalNamelist, world: int, *, halo: int | None = None,
                 boundary_pass: bool = False, copier=None, step_fn=None):
        H = halo_rows(nl) if halo is None else int(halo)
        self.slabs = [SlabStepper(nl, slab_layout(nl.ny, world, r, H), boundary_pass=boundary_pass, copier=copier,
                                  step_fn=step_fn) for r in range(world)]

    def load(self, carry: dycore.OperationalCarry) -> None:
        self._like = carry
        for s in self.slabs:
            s.load(carry)

    def step(self, lead_seconds) -> None:
        for s in self.slabs:
            s.advance(lead_seconds)
        self.exchange()

    def exchange(self) -> None:
        if len(self.slabs) == 1:
            return
        sent = [s.pack() for s in self.slabs]
        for s in self.slabs:
            L = s.layout
            s.unpack(sent[L.below][1], sent[L.above][0])

    def gather(self) -> dycore.OperationalCarry:
        out = _like_global(self._like)
        for s in self.slabs:
            s.owned_into(out)
        return out


class DistributedSlab:
    """This process's slab of a decomposition over a ``torch.distributed``
    group (one rank per GPU over NCCL; gloo for host tensors): each step
    advances the slab, then swaps halo blocks with the ranks below and above
    in one batch of point-to-point sends and receives."""

    def __init__(self, nl: dycore.OperationalNamelist, *, group=None, halo: int | None = None,
                 boundary_pass: bool = False, copier=None, step_fn=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        world = dist.get_world_size(group)
        rank = dist.get_rank(group)
        H = halo_rows(nl) if halo is None else int(halo)
        self.slab = SlabStepper(nl, slab_layout(nl.ny, world, rank, H), boundary_pass=boundary_pass,
                                copier=copier, step_fn=step_fn)

    def _global_rank(self, r: int) -> int:
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def load(self, carry: dycore.OperationalCarry) -> None:
        self._like = carry
        self.slab.load(carry)

    def step(self, lead_seconds) -> None:
        self.slab.advance(lead_seconds)
        self.exchange()

    def exchange(self) -> None:
        s, dist = self.slab, self.dist
        L = s.layout
        if L.world == 1:
            return
        to_below, to_above = s.pack()
        nb, na = s.recv_sizes()
        dev = to_below.device
        from_below = torch.empty(nb, dtype=torch.float64, device=dev)
        from_above = torch.empty(na, dtype=torch.float64, device=dev)
        below, above = self._global_rank(L.below), self._global_rank(L.above)
        # the upward flow (tag 0) first, then the downward flow (tag 1), on every
        # rank: with two ranks both neighbours are the same peer, and the
        # messages between a pair match in this order
        ops = [dist.P2POp(dist.isend, to_above, above, self.group, 0),
               dist.P2POp(dist.irecv, from_below, below, self.group, 0),
               dist.P2POp(dist.isend, to_below, below, self.group, 1),
               dist.P2POp(dist.irecv, from_above, above, self.group, 1)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        s.unpack(from_below, from_above)

    def gather(self) -> dycore.OperationalCarry:
        """The whole-domain carry on every rank (owned rows all-gathered)."""
        s, dist = self.slab, self.dist
        L = s.layout
        names = [n for n in dycore.State.__dataclass_fields__
                 if not n.endswith("_bdy") and getattr(s.carry.state, n) is not None]
        carry_names = [n for n in ("mudf", "t_2ave", "ww", "muave", "muts", "ph_tend", "u_save", "v_save", "w_save",
                                   "t_save", "ph_save", "mu_save", "ww_save") if getattr(s.carry, n) is not None]
        tensors = [getattr(s.carry.state, n) for n in names] + [getattr(s.carry, n) for n in carry_names]
        most = max(own_bounds(L.ny, L.world, r)[1] - own_bounds(L.ny, L.world, r)[0] for r in range(L.world))
        # one padded block per rank: every field's owned rows, plus one row for y-face arrays
        blocks, off = [], 0
        for n, t in zip(names + carry_names, tensors):
            t3 = _as3(t)
            extra = 1 if n in ("v", "v_save") and L.own_hi == L.ny else 0
            blocks.append((t, L.own_local, L.own + extra, off))
            off += t3.shape[0] * (most + 1) * t3.shape[2]
        buf = torch.zeros(off, dtype=torch.float64, device=tensors[0].device)
        s.copier.pack(blocks, buf)
        parts = [torch.empty_like(buf) for _ in range(L.world)]
        dist.all_gather(parts, buf, group=self.group)
        out = _like_global(self._like)
        for r, part in enumerate(parts):
            lo, hi = own_bounds(L.ny, L.world, r)
            rb, off = [], 0
            for n, t in zip(names + carry_names, tensors):
                t3 = _as3(t)
                dst = getattr(out.state, n) if n in names else getattr(out, n)
                extra = 1 if n in ("v", "v_save") and hi == L.ny else 0
                rb.append((dst, lo, hi - lo + extra, off))
                off += t3.shape[0] * (most + 1) * t3.shape[2]
            s.copier.unpack(rb, part)
        return out
