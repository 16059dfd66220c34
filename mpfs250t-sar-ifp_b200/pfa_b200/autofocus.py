"""Gradient-based phase autofocus over the B200 engine.

``entropy_grad(plan, signal, theta)`` calls ``pfa_autofocus_grad``: the float PFA image of
s[i,k] exp(-j theta_i), its entropy E and dE/dtheta from the hand-written adjoint kernels.
``ImageEntropy`` wraps it as a ``torch.autograd.Function`` (the forward computes the gradient too, so
backward only scales it), and ``autofocus`` runs plain gradient descent with a normalised step on theta;
``descent_step`` (``pfa_autofocus_step``) does one such step entirely on the device, and ``form_corrected``
(``pfa_form_float_phase``) forms the image of the corrected signal without a corrected copy.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .engine import FloatPlan, _stream_handle


def entropy_grad(plan: FloatPlan, signal, theta, dtheta=None, entropy=None, stream=None):
    """signal: (m, n) complex64 CUDA tensor; theta: (m,) float32 CUDA tensor.  Returns (E, dE/dtheta) as
    CUDA tensors (E float64 scalar tensor)."""
    import torch
    theta = theta.contiguous().float()
    dth = dtheta if dtheta is not None else torch.empty_like(theta)
    ent = entropy if entropy is not None else torch.empty((), dtype=torch.float64, device=theta.device)
    _lib.check(plan._lib.pfa_autofocus_grad(plan.handle, C.c_void_p(signal.data_ptr()), C.c_void_p(theta.data_ptr()),
                                            C.c_void_p(dth.data_ptr()), C.c_void_p(ent.data_ptr()),
                                            _stream_handle(stream)), plan.handle)
    return ent, dth


def descent_step(plan: FloatPlan, signal, theta, step: float, entropy=None, stream=None):
    """One descent step on the device (pfa_autofocus_step): theta <- theta - step (g - mean g) / max|g - mean g|
    in place, g = dE/dtheta.  No host synchronisation."""
    _lib.check(plan._lib.pfa_autofocus_step(plan.handle, C.c_void_p(signal.data_ptr()), C.c_void_p(theta.data_ptr()),
                                            C.c_float(step),
                                            C.c_void_p(entropy.data_ptr()) if entropy is not None else None,
                                            _stream_handle(stream)), plan.handle)
    return theta


def form_corrected(plan: FloatPlan, signal, theta, out=None, detect: str = "mag", stream=None):
    """Image of s[i, k] exp(-j theta_i) (pfa_form_float_phase: the correction is applied in pass 1)."""
    import torch
    dt = torch.complex64 if detect == "complex" else torch.float32
    img = out if out is not None else torch.empty((plan.m2, plan.n2), dtype=dt, device=signal.device)
    _lib.check(plan._lib.pfa_form_float_phase(plan.handle, C.c_void_p(signal.data_ptr()),
                                              C.c_void_p(theta.contiguous().data_ptr()), C.c_void_p(img.data_ptr()),
                                              plan.DETECT[detect], _stream_handle(stream)), plan.handle)
    return img


def _function():
    import torch

    class ImageEntropy(torch.autograd.Function):
        """E(theta) = entropy of |PFA(s exp(-j theta))|^2; backward returns dE/dtheta (no grad for s)."""

        @staticmethod
        def forward(ctx, theta, plan, signal):
            ent, dth = entropy_grad(plan, signal, theta.detach())
            ctx.save_for_backward(dth)
            return ent.to(theta.dtype)

        @staticmethod
        def backward(ctx, grad_out):
            (dth,) = ctx.saved_tensors
            return grad_out * dth, None, None

    return ImageEntropy


_IE = None


def image_entropy(theta, plan: FloatPlan, signal):
    global _IE
    if _IE is None:
        _IE = _function()
    return _IE.apply(theta, plan, signal)


def autofocus(plan: FloatPlan, signal, theta0=None, steps: int = 50, step: float = 0.5, history: bool = False):
    """Gradient descent on the per-pulse phase: theta <- theta - step * g / max|g| each iteration
    (g with its mean removed).  Returns (theta, entropies).  Without ``history`` every step runs on the
    device (pfa_autofocus_step); with it the entropy of each step is read back."""
    import torch
    m = plan.m
    theta = torch.zeros(m, dtype=torch.float32, device=signal.device) if theta0 is None else theta0.clone().float()
    dth = torch.empty_like(theta)
    ent = torch.empty((), dtype=torch.float64, device=signal.device)
    hist = []
    if not history:
        theta = theta.contiguous()
        for _ in range(steps):
            descent_step(plan, signal, theta, step)
        return theta, hist
    for _ in range(steps):
        entropy_grad(plan, signal, theta, dth, ent)
        if history:
            hist.append(float(ent))
        g = dth - dth.mean()                     # a constant phase does not change the image
        theta = theta - step * g / g.abs().max().clamp_min(1e-30)
    return theta, hist
