"""Differentiable Lomb-Scargle power and Newton refinement of its peaks.

No counterpart in the reference, which evaluates the LS power on the trial
period grid only (periodfind/ls.pyx:37-176, periodfind/cuda/ls.cu:75-136).
Here the same power (the reference's tau expression, written as the
equivalent closed form 0.5 v^T M^-1 v) is a function of the magnitudes and
of the angular frequency omega = 2 pi / period, with a hand-written backward
kernel behind `torch.autograd.Function`:

    power = ls_power(times, mags, omega, offsets)       # [n_curves, n_freq]
    power.sum().backward()                               # mags.grad, omega.grad

Curves are CSR: `times` and `mags` are 1-D float32 CUDA tensors holding all
curves back to back, `offsets` a host int64 array of n_curves + 1 entries.
`omega` is a float64 CUDA tensor, [n_freq] (one grid for every curve) or
[n_curves, n_freq].  Derivatives are FP32 sums; the phase is reduced in FP64.

`refine_peaks` runs safeguarded Newton steps on dP/domega inside a bracket
around each start frequency (one kernel launch for all steps) and returns
the refined frequencies and powers.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native as nat


def _host_offsets(offsets, total: int) -> np.ndarray:
    if isinstance(offsets, torch.Tensor):
        offsets = offsets.detach().cpu().numpy()
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    if off.ndim != 1 or len(off) < 1:
        raise ValueError("offsets must be a 1-D array of n_curves + 1 entries")
    if off[0] != 0 or off[-1] != total or np.any(np.diff(off) < 0):
        raise ValueError("offsets must start at 0, be non-decreasing and end at len(times)")
    return off


def _cuda_f32(x: torch.Tensor, name: str) -> torch.Tensor:
    if not isinstance(x, torch.Tensor) or not x.is_cuda or x.dtype != torch.float32:
        raise TypeError(f"{name} must be a float32 CUDA tensor")
    if x.dim() != 1:
        raise ValueError(f"{name} must be 1-D (curves back to back)")
    return x.contiguous()


def _omega(omega: torch.Tensor, n_curves: int):
    if not isinstance(omega, torch.Tensor) or not omega.is_cuda:
        raise TypeError("omega must be a CUDA tensor")
    w = omega.detach().to(torch.float64).contiguous()
    if w.dim() == 1:
        return w, 0, w.shape[0]
    if w.dim() == 2 and w.shape[0] == n_curves:
        return w, w.shape[1], w.shape[1]
    raise ValueError("omega must be [n_freq] or [n_curves, n_freq]")


def _stream(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


class LombScarglePower(torch.autograd.Function):
    """power[c, k] = LS power of curve c at angular frequency omega[(c,) k]."""

    @staticmethod
    def forward(ctx, times, mags, omega, offsets):
        t = _cuda_f32(times, "times")
        y = _cuda_f32(mags.detach(), "mags")
        if t.shape != y.shape or t.device != y.device:
            raise ValueError("times and mags must have the same shape and device")
        off = _host_offsets(offsets, t.shape[0])
        n_curves = len(off) - 1
        w, stride, K = _omega(omega, n_curves)
        dev = t.device
        power = torch.empty((n_curves, K), dtype=torch.float32, device=dev)
        dpdw = torch.empty_like(power)
        coef = torch.empty((n_curves, K, 2), dtype=torch.float32, device=dev)
        c = nat.default_context(dev.index or 0)
        with c.lock:
            c.check(c.lib.pf_ls_eval_dev(c.handle, t.data_ptr(), y.data_ptr(), off.ctypes.data,
                                         n_curves, w.data_ptr(), stride, K, power.data_ptr(),
                                         dpdw.data_ptr(), None, coef.data_ptr(), _stream(dev)))
        ctx.save_for_backward(t, w, dpdw, coef)
        ctx.off = off
        ctx.stride = stride
        ctx.omega_shape = tuple(omega.shape)
        ctx.omega_dtype = omega.dtype
        ctx.mark_non_differentiable(dpdw)
        return power

    @staticmethod
    def backward(ctx, grad_power):
        t, w, dpdw, coef = ctx.saved_tensors
        need_mags, need_omega = ctx.needs_input_grad[1], ctx.needs_input_grad[2]
        grad_mags = grad_omega = None
        if not (need_mags or need_omega):
            return None, None, None, None
        off = ctx.off
        n_curves = len(off) - 1
        K = coef.shape[1]
        g = grad_power.detach().to(torch.float32).contiguous()
        dev = t.device
        gm = torch.empty_like(t) if need_mags else None
        gw = torch.empty((n_curves, K), dtype=torch.float64, device=dev) if need_omega else None
        c = nat.default_context(dev.index or 0)
        with c.lock:
            c.check(c.lib.pf_ls_backward_dev(
                c.handle, t.data_ptr(), off.ctypes.data, n_curves, w.data_ptr(), ctx.stride, K,
                g.data_ptr(), dpdw.data_ptr(), coef.data_ptr(),
                gw.data_ptr() if gw is not None else None,
                gm.data_ptr() if gm is not None else None, _stream(dev)))
        if need_mags:
            grad_mags = gm
        if need_omega:
            grad_omega = (gw.sum(0) if len(ctx.omega_shape) == 1 else gw).to(ctx.omega_dtype)
        return None, grad_mags, grad_omega, None


def ls_power(times, mags, omega, offsets):
    """Differentiable LS power [n_curves, n_freq] (see the module docstring)."""
    return LombScarglePower.apply(times, mags, omega, offsets)


def ls_derivatives(times, mags, omega, offsets, second=True):
    """(power, dP/domega, d2P/domega2 or None, coef [.., 2]) without autograd."""
    t = _cuda_f32(times, "times")
    y = _cuda_f32(mags, "mags")
    off = _host_offsets(offsets, t.shape[0])
    n_curves = len(off) - 1
    w, stride, K = _omega(omega, n_curves)
    dev = t.device
    power = torch.empty((n_curves, K), dtype=torch.float32, device=dev)
    d1 = torch.empty_like(power)
    d2 = torch.empty_like(power) if second else None
    coef = torch.empty((n_curves, K, 2), dtype=torch.float32, device=dev)
    c = nat.default_context(dev.index or 0)
    with c.lock:
        c.check(c.lib.pf_ls_eval_dev(c.handle, t.data_ptr(), y.data_ptr(), off.ctypes.data,
                                     n_curves, w.data_ptr(), stride, K, power.data_ptr(),
                                     d1.data_ptr(), d2.data_ptr() if second else None,
                                     coef.data_ptr(), _stream(dev)))
    return power, d1, d2, coef


def refine_peaks(times, mags, omega0, half_width, offsets, n_steps=5):
    """Newton-refine LS maxima.  omega0, half_width: float64 CUDA tensors
    [n_curves, K] (start frequency and bracket half-width, rad / time unit).
    Returns (omega float64 [n_curves, K], power float32 [n_curves, K])."""
    t = _cuda_f32(times, "times")
    y = _cuda_f32(mags, "mags")
    off = _host_offsets(offsets, t.shape[0])
    n_curves = len(off) - 1
    w0 = omega0.detach().to(torch.float64).contiguous()
    hw = half_width.detach().to(device=w0.device, dtype=torch.float64).contiguous()
    if w0.dim() != 2 or w0.shape[0] != n_curves or hw.shape != w0.shape:
        raise ValueError("omega0 and half_width must both be [n_curves, K]")
    K = w0.shape[1]
    w = torch.empty_like(w0)
    power = torch.empty(w0.shape, dtype=torch.float32, device=w0.device)
    c = nat.default_context(t.device.index or 0)
    with c.lock:
        c.check(c.lib.pf_ls_refine_dev(c.handle, t.data_ptr(), y.data_ptr(), off.ctypes.data,
                                       n_curves, w0.data_ptr(), hw.data_ptr(), K,
                                       int(n_steps), w.data_ptr(), power.data_ptr(),
                                       _stream(t.device)))
    return w, power
