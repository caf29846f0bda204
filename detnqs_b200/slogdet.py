"""Batched sign and log|det| of small real matrices on the GPU.

Mirrors detnqs/models/slogdet.py's fused kernel path (``slogdet(A,
use_fast_kernel=True)``: forward by LU with partial pivoting, gradient of
log|det| as A^{-T}) over ``dnq_slogdet`` / ``dnq_slogdet_grad``.  Where the
reference wires the kernels into JAX with ``jax.custom_vjp``,
``SlogdetFunction`` wires them into torch autograd.
"""

from __future__ import annotations

from functools import lru_cache

import numpy as np

from . import native as N


def _check(a):
    is_t = hasattr(a, "is_cuda")
    dt = str(a.dtype).replace("torch.", "")
    if dt not in ("float32", "float64"):
        raise TypeError(f"Unsupported dtype {a.dtype}")
    if a.ndim < 2 or a.shape[-1] != a.shape[-2]:
        raise ValueError(f"Expected square matrix, got shape {tuple(a.shape)}")
    n = int(a.shape[-1])
    if not (2 <= n <= 64):
        raise ValueError(f"Matrix size {n} outside [2, 64] range")
    prec = N.F64 if dt == "float64" else N.F32
    return is_t, n, prec


def _device_of(a, device):
    if hasattr(a, "is_cuda") and a.is_cuda:
        return a.device.index if a.device.index is not None else device
    return device


def slogdet(a, device: int = 0):
    """(sign, logabsdet) of a (..., n, n) float32/float64 array or tensor,
    2 <= n <= 64; results have the batch shape and a's type.  Host arrays
    give numpy results, CUDA tensors give CUDA tensors."""
    is_t, n, prec = _check(a)
    batch = tuple(a.shape[:-2])
    if is_t:
        import torch
        x = a.contiguous()
        sign = torch.empty(batch, dtype=a.dtype, device=a.device)
        logabs = torch.empty(batch, dtype=a.dtype, device=a.device)
    else:
        x = np.ascontiguousarray(a)
        sign = np.empty(batch, x.dtype)
        logabs = np.empty(batch, x.dtype)
    B = int(np.prod(batch)) if batch else 1
    N.check(N.lib.dnq_slogdet(N.ptr(x), B, n, prec, N.ptr(sign), N.ptr(logabs),
                              int(_device_of(a, device)), N.stream_of(x)))
    return sign, logabs


def slogdet_grad(a, cot_logabs, device: int = 0):
    """cot_logabs * A^{-T} for every matrix of a (the gradient of
    log|det|); zero for a matrix whose factorisation meets a zero pivot."""
    is_t, n, prec = _check(a)
    batch = tuple(a.shape[:-2])
    if tuple(cot_logabs.shape) != batch:
        raise ValueError("Batch shape mismatch")
    if is_t:
        import torch
        x = a.contiguous()
        c = cot_logabs.to(a.dtype).contiguous()
        g = torch.empty_like(x)
    else:
        x = np.ascontiguousarray(a)
        c = np.ascontiguousarray(cot_logabs, dtype=x.dtype)
        g = np.empty_like(x)
    B = int(np.prod(batch)) if batch else 1
    N.check(N.lib.dnq_slogdet_grad(N.ptr(x), N.ptr(c), B, n, prec, N.ptr(g),
                                   int(_device_of(a, device)), N.stream_of(x, c)))
    return g


@lru_cache(maxsize=None)
def _autograd():
    import torch

    class SlogdetFunction(torch.autograd.Function):
        """(sign, logabsdet) with the gradient of logabsdet; sign carries
        none (the reference's _fused_logdet custom VJP, slogdet.py:103-154)."""

        @staticmethod
        def forward(ctx, a):
            ctx.save_for_backward(a)
            return slogdet(a)

        @staticmethod
        def backward(ctx, g_sign, g_logabs):
            (a,) = ctx.saved_tensors
            if g_logabs is None:
                return None
            return slogdet_grad(a, g_logabs)

    return SlogdetFunction


def slogdet_autograd(a):
    """slogdet of a CUDA tensor that torch autograd differentiates."""
    return _autograd().apply(a)


__all__ = ["slogdet", "slogdet_grad", "slogdet_autograd"]
