"""Residual energy of a fixed spike assignment and its adjoint (template refinement).

No counterpart in the reference: after a pursuit has fixed which template fires
where, the templates (and per-spike amplitudes and sub-sample shifts) can be
refined by gradient descent on the residual energy

    E = sum_{c,x} (v[c, x] - sum_k a_k * shift(T_{l_k}, tau_k)[c, x - s_k])^2

with linear interpolation for the fractional shift (``include/fbp.h``,
``fbp_adjoint_loss``).  ``residual_energy`` is a ``torch.autograd.Function``
whose forward and backward are the hand-written CUDA kernels of
``csrc/adjoint.cu``: the backward recomputes each spike's residual tile instead
of keeping anything from the forward.  Sums run in FP64 on the device.

    loss = residual_energy(voltage, templates, spike_idx, spike_lab, amplitude, shift)
    loss.backward()     # templates.grad, amplitude.grad, shift.grad
"""
from __future__ import annotations

import ctypes

import torch

from . import _native


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None


def _stream(t):
    # the kernels run on torch's current stream of the tensor's device, in order
    # with the work that produced their inputs and the work that reads their outputs
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


class _ResidualEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, voltage, templates, spike_idx, spike_lab, amplitude, shift):
        C, N = voltage.shape
        M = templates.shape[0]
        W = templates.numel() // (M * C)
        # spikes in onset order (the kernels find overlapping neighbours by binary search)
        order = torch.argsort(spike_idx.to(torch.int64), stable=True)
        idx = spike_idx.to(torch.int64)[order].to(torch.int32).contiguous()
        lab = spike_lab.to(torch.int64)[order].to(torch.int32).contiguous()
        amp = amplitude.detach()[order].to(torch.float32).contiguous()
        tau = shift.detach()[order].to(torch.float32).contiguous()
        V = voltage.detach().to(torch.float32).contiguous()
        T = templates.detach().to(torch.float32).reshape(M, C * W).contiguous()
        d = _native.dims(C, N, M, W, 0)
        loss = torch.zeros(1, dtype=torch.float64, device=voltage.device)
        _native.check(_native.lib().fbp_adjoint_loss(ctypes.byref(d), _ptr(V), _ptr(T), _ptr(idx), _ptr(lab),
                                                     _ptr(amp), _ptr(tau), int(idx.numel()), _ptr(loss),
                                                     _stream(V)))
        ctx.save_for_backward(V, T, idx, lab, amp, tau, order)
        ctx.shape = (C, N, M, W)
        ctx.t_shape, ctx.t_dtype = templates.shape, templates.dtype
        ctx.a_dtype, ctx.s_dtype = amplitude.dtype, shift.dtype
        return loss[0].to(torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        V, T, idx, lab, amp, tau, order = ctx.saved_tensors
        C, N, M, W = ctx.shape
        n = idx.numel()
        d = _native.dims(C, N, M, W, 0)
        g64 = torch.empty(M * C * W, dtype=torch.float64, device=V.device)
        gT = torch.empty(M * C * W, dtype=torch.float32, device=V.device)
        ga = torch.empty(n, dtype=torch.float32, device=V.device)
        gs = torch.empty(n, dtype=torch.float32, device=V.device)
        scale = float(grad_out.item())
        _native.check(_native.lib().fbp_adjoint_grad(ctypes.byref(d), _ptr(V), _ptr(T), _ptr(idx), _ptr(lab),
                                                     _ptr(amp), _ptr(tau), int(n), ctypes.c_double(scale),
                                                     _ptr(g64), _ptr(gT), _ptr(ga), _ptr(gs), _stream(V)))
        inv = torch.empty_like(order)
        inv[order] = torch.arange(n, device=order.device)
        grad_T = gT.reshape(ctx.t_shape).to(ctx.t_dtype) if ctx.needs_input_grad[1] else None
        grad_a = ga[inv].to(ctx.a_dtype) if ctx.needs_input_grad[4] else None
        grad_s = gs[inv].to(ctx.s_dtype) if ctx.needs_input_grad[5] else None
        return None, grad_T, None, None, grad_a, grad_s


def residual_energy(voltage: torch.Tensor, templates: torch.Tensor, spike_idx: torch.Tensor,
                    spike_lab: torch.Tensor, amplitude: torch.Tensor, shift: torch.Tensor) -> torch.Tensor:
    """FP64 residual energy of a fixed assignment; differentiable in templates, amplitude, shift.

    voltage    [C, N] float32, CUDA
    templates  [M, C*W] or [M, C, W] float32, CUDA
    spike_idx  [n] integer onsets (template sample 0 lands on voltage sample spike_idx[k])
    spike_lab  [n] integer template rows
    amplitude  [n] float32, shift [n] float32 in (-1, 1) samples
    """
    if not voltage.is_cuda:
        raise RuntimeError("No GPU available")
    return _ResidualEnergy.apply(voltage, templates, spike_idx, spike_lab, amplitude, shift)
