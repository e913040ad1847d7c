"""Differentiable scalar advection: the CUDA h5/v3 flux-form operator with its
hand-written adjoint behind ``torch.autograd.Function``.

``scalar_advection(q, ru, rv, rom, namelist)`` returns the advective
tendency of ``q`` (``advect_scalar_flux``, dynamics/flux_advection.py:482-568,
doubly periodic) for fixed transport velocities; ``backward`` applies the
adjoint kernel (``wrfgpu_scalar_advection_adjoint``) to the incoming
gradient, so gradients flow to ``q`` (the velocities are treated as
constants: their gradient is not built).
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


class ScalarAdvection(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, ru, rv, rom, op: _Op):
        q, ru, rv, rom = (t.contiguous() for t in (q, ru, rv, rom))
        tend = torch.empty_like(q)
        op.apply("wrfgpu_scalar_advection", q, ru, rv, rom, tend)
        ctx.save_for_backward(ru, rv, rom)
        ctx.op = op
        return tend

    @staticmethod
    def backward(ctx, tend_bar):
        ru, rv, rom = ctx.saved_tensors
        if any(ctx.needs_input_grad[1:4]):
            raise NotImplementedError("gradients with respect to the transport velocities are not built")
        q_bar = torch.empty_like(tend_bar)
        ctx.op.apply("wrfgpu_scalar_advection_adjoint", tend_bar.contiguous(), ru, rv, rom, q_bar)
        return q_bar, None, None, None, None


def scalar_advection(q: torch.Tensor, ru: torch.Tensor, rv: torch.Tensor, rom: torch.Tensor,
                     namelist: dycore.OperationalNamelist) -> torch.Tensor:
    """Flux-form advective tendency of ``q`` (nz, ny, nx) for transport
    velocities ``ru``, ``rv`` (nz, ny, nx) and ``rom`` (nz+1, ny, nx);
    differentiable with respect to ``q``."""
    return ScalarAdvection.apply(q, ru, rv, rom, _Op(namelist))
