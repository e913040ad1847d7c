"""Hand-written adjoints behind ``torch.autograd.Function``.

* ``scalar_advection(q, ru, rv, rom, namelist)`` returns the advective
  tendency of ``q`` (``advect_scalar_flux``, dynamics/flux_advection.py:482-568,
  doubly periodic), ``advect_u`` / ``advect_v`` / ``advect_w`` those of the
  momentum components (``advect_u_flux`` / ``advect_v_flux`` /
  ``advect_w_flux``, :1131-1329, periodic);
  ``backward`` applies the hand-written VJP kernel
  (``wrfgpu_flux_advection_vjp``, one launch) for the advected field and the
  transport velocities ``ru``, ``rv``, ``rom`` (the operator is bilinear; the
  upwind switches are held at their forward sign), with w's vertical part
  through ``wrfgpu_w_vertical_advection_vjp``.
* ``acoustic_substep(work, op)`` / ``acoustic_loop(work, op, nsub)``: one or
  ``nsub`` acoustic small steps (acoustic_substep_core, core/acoustic.py:
  837-1150) of the evolving work state for fixed stage constants, with the
  VJP kernels of ``wrfgpu_acoustic_substep_vjp`` in the backward pass; the
  loop keeps one checkpoint and recomputes its substeps.
"""

from __future__ import annotations

import ctypes

import torch

from . import _capi, dycore


class _Op:
    """Params and metrics structs of one namelist (no workspace)."""

    def __init__(self, nl: dycore.OperationalNamelist):
        self.nl = nl
        self.params = dycore.step_params(nl)
        _capi.check(_capi.load().wrfgpu_step_params_validate(ctypes.byref(self.params)))
        self.metrics = _capi.Metrics(*[dycore._ptr(getattr(nl.metrics, n)) for n in dycore.METRIC_ARRAYS])

    def apply(self, fn_name, src, ru, rv, rom, dst):
        lib = _capi.load()
        st = torch.cuda.current_stream(src.device)
        _capi.check(getattr(lib, fn_name)(ctypes.byref(self.params), ctypes.byref(self.metrics),
                                          ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(ru.data_ptr()),
                                          ctypes.c_void_p(rv.data_ptr()), ctypes.c_void_p(rom.data_ptr()),
                                          ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(st.cuda_stream)))


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else None)


class FluxAdvection(torch.autograd.Function):
    """The flux-form advection operator ``wrfgpu_flux_advection`` with its
    map-factor weights ``hfac`` / ``vfac`` (constants, not differentiated)."""

    @staticmethod
    def forward(ctx, q, ru, rv, rom, op: _Op, hfac, vfac):
        # rom None: the horizontal flux divergence alone
        q, ru, rv, rom = (t.contiguous() if t is not None else None for t in (q, ru, rv, rom))
        tend = torch.empty_like(q)
        st = torch.cuda.current_stream(q.device)
        _capi.check(_capi.load().wrfgpu_flux_advection(
            ctypes.byref(op.params), ctypes.byref(op.metrics), _ptr(q), _ptr(ru), _ptr(rv), _ptr(rom), _ptr(hfac),
            _ptr(vfac), _ptr(tend), ctypes.c_void_p(st.cuda_stream)))
        ctx.save_for_backward(q, ru, rv, rom)
        ctx.op, ctx.hfac, ctx.vfac = op, hfac, vfac
        return tend

    @staticmethod
    def backward(ctx, tend_bar):
        q, ru, rv, rom = ctx.saved_tensors
        need = ctx.needs_input_grad[:4]
        outs = [torch.empty_like(t) if n else None for t, n in zip((q, ru, rv, rom), need)]
        if any(o is not None for o in outs):
            # the field's and the velocities' cotangents in one launch
            st = torch.cuda.current_stream(q.device)
            _capi.check(_capi.load().wrfgpu_flux_advection_vjp(
                ctypes.byref(ctx.op.params), ctypes.byref(ctx.op.metrics), _ptr(q), _ptr(tend_bar.contiguous()),
                _ptr(ru), _ptr(rv), _ptr(rom), _ptr(ctx.hfac), _ptr(ctx.vfac), *map(_ptr, outs),
                ctypes.c_void_p(st.cuda_stream)))
        return (*outs, None, None, None)


def scalar_advection(q: torch.Tensor, ru: torch.Tensor, rv: torch.Tensor, rom: torch.Tensor,
                     namelist: dycore.OperationalNamelist) -> torch.Tensor:
    """Flux-form advective tendency of ``q`` (nz, ny, nx) for transport
    velocities ``ru``, ``rv`` (nz, ny, nx) and ``rom`` (nz+1, ny, nx);
    differentiable with respect to ``q`` and the velocities."""
    return FluxAdvection.apply(q, ru, rv, rom, _Op(namelist), None, None)


def advect_u(u: torch.Tensor, ru: torch.Tensor, rv: torch.Tensor, rom: torch.Tensor,
             namelist: dycore.OperationalNamelist) -> torch.Tensor:
    """advect_u_flux (dynamics/flux_advection.py:1131-1202), doubly periodic:
    the advective tendency of u (nz, ny, nx+1) for the transport velocities
    ru, rv (nz, ny, nx) and rom (nz+1, ny, nx) -- the operator on u's core
    faces with the velocities averaged to them and the map factor msfux; the
    wrap face repeats face 0.  Differentiable with respect to u (its wrap
    face does not enter) and the velocities."""
    m = namelist.metrics
    nx = ru.shape[-1]
    velx = 0.5 * (ru + torch.roll(ru, 1, -1))
    vely = 0.5 * (rv + torch.roll(rv, 1, -1))
    velz = 0.5 * (rom + torch.roll(rom, 1, -1))
    tend = FluxAdvection.apply(u[..., :nx], velx, vely, velz, _Op(namelist), m.msfux[:, :nx].contiguous(), None)
    return torch.cat((tend, tend[:, :, :1]), dim=2)


def advect_v(v: torch.Tensor, ru: torch.Tensor, rv: torch.Tensor, rom: torch.Tensor,
             namelist: dycore.OperationalNamelist) -> torch.Tensor:
    """advect_v_flux (dynamics/flux_advection.py:1205-1274), doubly periodic:
    the advective tendency of v (nz, ny+1, nx) -- the operator on v's core
    faces with the velocities averaged to them, the map factor msfvy and the
    vertical term scaled by msfvy / msfvx; the wrap row repeats row 0."""
    m = namelist.metrics
    ny = rv.shape[-2]
    velx = 0.5 * (ru + torch.roll(ru, 1, -2))
    vely = 0.5 * (rv + torch.roll(rv, 1, -2))
    velz = 0.5 * (rom + torch.roll(rom, 1, -2))
    hfac = m.msfvy[:ny].contiguous()
    vfac = (m.msfvy[:ny] / m.msfvx[:ny]).contiguous()
    tend = FluxAdvection.apply(v[:, :ny, :], velx, vely, velz, _Op(namelist), hfac, vfac)
    return torch.cat((tend, tend[:, :1, :]), dim=1)


class _WVertical(torch.autograd.Function):
    """The vertical flux divergence of w (``wrfgpu_w_vertical_advection``)
    and its VJP (``wrfgpu_w_vertical_advection_vjp``)."""

    @staticmethod
    def forward(ctx, w, rom, op: _Op):
        w, rom = w.contiguous(), rom.contiguous()
        tend = torch.empty_like(w)
        st = torch.cuda.current_stream(w.device)
        _capi.check(_capi.load().wrfgpu_w_vertical_advection(
            ctypes.byref(op.params), ctypes.byref(op.metrics), _ptr(w), _ptr(rom), _ptr(tend),
            ctypes.c_void_p(st.cuda_stream)))
        ctx.save_for_backward(w, rom)
        ctx.op = op
        return tend

    @staticmethod
    def backward(ctx, tend_bar):
        w, rom = ctx.saved_tensors
        outs = [torch.empty_like(t) if n else None for t, n in zip((w, rom), ctx.needs_input_grad[:2])]
        if any(o is not None for o in outs):
            st = torch.cuda.current_stream(w.device)
            _capi.check(_capi.load().wrfgpu_w_vertical_advection_vjp(
                ctypes.byref(ctx.op.params), ctypes.byref(ctx.op.metrics), _ptr(w), _ptr(rom),
                _ptr(tend_bar.contiguous()), *map(_ptr, outs), ctypes.c_void_p(st.cuda_stream)))
        return (*outs, None)


def _mass_to_full(f, fnm, fnp):
    """flux_advection.py:1332-1352: a mass-level field on the w levels."""
    inner = fnm[1:, None, None] * f[1:] + fnp[1:, None, None] * f[:-1]
    return torch.cat((f[:1], inner, f[-1:]), dim=0)


def advect_w(w: torch.Tensor, ru: torch.Tensor, rv: torch.Tensor, rom: torch.Tensor,
             namelist: dycore.OperationalNamelist) -> torch.Tensor:
    """advect_w_flux (dynamics/flux_advection.py:1277-1329), doubly periodic:
    the advective tendency of w (nz+1, ny, nx) -- the horizontal flux
    operator on w's levels with ru, rv interpolated to them (map factor
    msftx) plus w's own vertical flux divergence by rom (namelist.top_lid).
    Differentiable with respect to w and the velocities."""
    m = namelist.metrics
    nz = ru.shape[0]
    fnm, fnp = m.fnm[:nz], m.fnp[:nz]
    ru_w, rv_w = _mass_to_full(ru, fnm, fnp), _mass_to_full(rv, fnm, fnp)
    op_w = _Op(namelist)
    op_w.params.nz = nz + 1  # the horizontal operator over w's levels
    tend_h = FluxAdvection.apply(w, ru_w, rv_w, None, op_w, m.msftx.contiguous(), None)
    return tend_h + _WVertical.apply(w, rom, _Op(namelist))


class AcousticOp:
    """One acoustic small step (``wrfgpu_acoustic_substep``) and its
    vector-Jacobian product (``wrfgpu_acoustic_substep_vjp``) for fixed stage
    constants: the reference's acoustic_substep_core (core/acoustic.py:837-1150)
    on a doubly periodic or specified domain (``u_target`` / ``v_target``
    given with run_boundary).  ``consts`` maps the names of
    ``_capi.ACOUSTIC_CONST_FIELDS`` to device tensors (``mu_tend`` may be
    absent); they are held for the op's lifetime."""

    def __init__(self, nl: dycore.OperationalNamelist, consts: dict, dts: float, device="cuda"):
        self.lib = _capi.load()
        self.nl = nl  # holds the metric tensors the metrics struct points into
        self.params = dycore.step_params(nl)
        _capi.check(self.lib.wrfgpu_step_params_validate(ctypes.byref(self.params)))
        self.metrics = _capi.Metrics(*[dycore._ptr(getattr(nl.metrics, n)) for n in dycore.METRIC_ARRAYS])
        self.consts_t = {n: t.contiguous() for n, t in consts.items() if t is not None}
        self.consts = _capi.AcousticConsts(*[dycore._ptr(self.consts_t.get(n)) for n in _capi.ACOUSTIC_CONST_FIELDS])
        n = ctypes.c_size_t(0)
        _capi.check(self.lib.wrfgpu_acoustic_workspace_size(ctypes.byref(self.params), ctypes.byref(n)))
        self.workspace = torch.empty(int(n.value), dtype=torch.uint8, device=device)
        self.dts = float(dts)

    @staticmethod
    def _work(ts) -> _capi.AcousticWork:
        return _capi.AcousticWork(*[dycore._ptr(t) for t in ts])

    def forward_(self, xs) -> None:
        """Advance the 14 work tensors (``_capi.ACOUSTIC_WORK_FIELDS`` order) one substep in place."""
        w = self._work(xs)
        st = torch.cuda.current_stream(xs[0].device)
        _capi.check(self.lib.wrfgpu_acoustic_substep(
            ctypes.byref(self.params), ctypes.byref(self.metrics), ctypes.byref(self.consts), ctypes.byref(w),
            self.dts, ctypes.c_void_p(self.workspace.data_ptr()), self.workspace.numel(),
            ctypes.c_void_p(st.cuda_stream)))

    def vjp(self, xs, cot_out, x_out=None, tendencies=False):
        """Cotangents of the 14 inputs ``xs`` from those of the outputs;
        ``x_out`` (the substep's outputs from ``xs``) is recomputed if None.
        With ``tendencies``, also returns the cotangents of the stage
        tendencies (a dict over ``_capi.ACOUSTIC_TEND_FIELDS``)."""
        cot_in = [torch.empty_like(t) for t in xs]
        st = torch.cuda.current_stream(xs[0].device)
        x, co, ci = self._work(xs), self._work(cot_out), self._work(cot_in)
        xo = ctypes.byref(self._work(x_out)) if x_out is not None else None
        tend, tc = None, None
        if tendencies:
            tend = {n: torch.empty_like(self.consts_t[n]) if n in self.consts_t
                    else torch.empty_like(self.consts_t["mut"]) for n in _capi.ACOUSTIC_TEND_FIELDS}
            tc = ctypes.byref(_capi.AcousticTendCot(*[dycore._ptr(tend[n]) for n in _capi.ACOUSTIC_TEND_FIELDS]))
        _capi.check(self.lib.wrfgpu_acoustic_substep_vjp(
            ctypes.byref(self.params), ctypes.byref(self.metrics), ctypes.byref(self.consts), ctypes.byref(x),
            xo, ctypes.byref(co), ctypes.byref(ci), tc, self.dts, ctypes.c_void_p(self.workspace.data_ptr()),
            self.workspace.numel(), ctypes.c_void_p(st.cuda_stream)))
        return (cot_in, tend) if tendencies else cot_in


class AcousticSubstep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, op: AcousticOp, *xs):
        x_in = [t.contiguous() for t in xs]
        out = [t.clone() for t in x_in]
        op.forward_(out)
        ctx.op = op
        ctx.save_for_backward(*x_in, *out)
        return tuple(out)

    @staticmethod
    def backward(ctx, *grads):
        saved = ctx.saved_tensors
        x_in, x_out = saved[:14], saved[14:]
        co = [g.contiguous() if g is not None else torch.zeros_like(x) for g, x in zip(grads, x_out)]
        return (None, *ctx.op.vjp(list(x_in), co, list(x_out)))


class AcousticLoop(torch.autograd.Function):
    """``nsub`` acoustic substeps behind one checkpoint: the forward keeps only
    the loop's input state; the backward recomputes the substep states from it
    (one forward pass) and applies the substep VJPs in reverse, each with its
    stored forward output."""

    @staticmethod
    def forward(ctx, op: AcousticOp, nsub: int, *xs):
        x0 = [t.contiguous() for t in xs]
        cur = [t.clone() for t in x0]
        for _ in range(nsub):
            op.forward_(cur)
        ctx.op, ctx.nsub = op, nsub
        ctx.save_for_backward(*x0)
        return tuple(cur)

    @staticmethod
    def backward(ctx, *grads):
        x0 = list(ctx.saved_tensors)
        states = [x0]
        for _ in range(ctx.nsub):
            nxt = [t.clone() for t in states[-1]]
            ctx.op.forward_(nxt)
            states.append(nxt)
        co = [g.contiguous() if g is not None else torch.zeros_like(x) for g, x in zip(grads, states[-1])]
        for n in range(ctx.nsub - 1, -1, -1):
            co = ctx.op.vjp(states[n], co, states[n + 1])
        return (None, None, *co)


def acoustic_loop(work: dict, op: AcousticOp, nsub: int) -> dict:
    """``nsub`` differentiable acoustic small steps with the loop input as the
    only stored state (substeps recomputed in the backward pass)."""
    names = _capi.ACOUSTIC_WORK_FIELDS
    outs = AcousticLoop.apply(op, int(nsub), *[work[n] for n in names])
    return dict(zip(names, outs))


def acoustic_substep(work: dict, op: AcousticOp) -> dict:
    """One differentiable acoustic small step of the work state ``work``
    (``_capi.ACOUSTIC_WORK_FIELDS`` names to tensors); gradients flow to every
    work field through the hand-written VJP kernels."""
    names = _capi.ACOUSTIC_WORK_FIELDS
    outs = AcousticSubstep.apply(op, *[work[n] for n in names])
    return dict(zip(names, outs))
