"""Determinants of up to 128 orbitals (two uint64 words per spin string).

The reference stores a spin string in one uint64 and stops at 64 orbitals
(``csrc/detnqs/determinant/det.hpp:30-36``, ``integral_mo.cpp:26-28``).
This module gives the same screened build for wider determinants, laid out
as ``uint64[N, 4] = (alpha lo, alpha hi, beta lo, beta hi)`` and ordered by
alpha as a 128-bit integer, then beta:

* :class:`IntCtxWide` -- integral context for up to 128 orbitals;
* :func:`get_ham_diag_wide` -- diagonal elements;
* :func:`get_ham_conn_wide` / :func:`get_ham_conn_amp_wide` -- the
  reference's ``get_ham_conn`` (static heat-bath) and ``get_ham_conn_amp``
  (dynamic amplitude screening) in its dict format;
* :func:`build_wide` -- the same blocks kept on the device, ready for
  ``H.spmv`` / ``H.proxy_spmv`` and :func:`ham_eff_wide` (downfolding).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N
from .core import IntCtx
from .device import DeviceHamiltonian, _f64


def _dets4(x):
    if hasattr(x, "data_ptr"):
        if x.dim() != 2 or x.shape[1] != 4:
            raise ValueError("two-word determinants must be uint64[N, 4]")
        return x.contiguous()
    a = np.ascontiguousarray(x, dtype=np.uint64)
    if a.ndim != 2 or a.shape[1] != 4:
        raise ValueError("two-word determinants must be uint64[N, 4]")
    return a


class IntCtxWide(IntCtx):
    """Integral context for up to 128 orbitals (packed arrays in the
    reference layout).  Accepted by the two-word functions only."""

    def __init__(self, *a, **k):
        raise TypeError("use IntCtxWide.from_arrays")

    @classmethod
    def from_arrays(cls, num_orb: int, h1e, eri, e_nuc: float, device: int = 0) -> "IntCtxWide":
        obj = cls.__new__(cls)
        h1 = np.ascontiguousarray(h1e, np.float64)
        er = np.ascontiguousarray(eri, np.float64)
        n1 = num_orb * (num_orb + 1) // 2
        if h1.size != n1 or er.size != n1 * (n1 + 1) // 2:
            raise ValueError("packed integral arrays have the wrong length")
        h = C.c_void_p()
        N.check(N.lib.dnq_ctx_create_wide(int(num_orb), h1.ctypes.data, er.ctypes.data,
                                          float(e_nuc), int(device), C.byref(h)))
        obj._h = h
        obj.n_orb = int(num_orb)
        obj.device = int(device)
        return obj


def get_ham_diag_wide(dets, ctx: IntCtx) -> np.ndarray:
    d = _dets4(dets)
    n = d.shape[0]
    out = np.empty(n, np.float64)
    N.check(N.lib.dnq_wide_diag(ctx.handle, N.ptr(d), n, out.ctypes.data, N.stream_of(d)))
    return out


def build_wide(ctx: IntCtx, dets, psi=None, *, n_orb: int, eps1: float) -> DeviceHamiltonian:
    """Device-resident H_VV, H_VP and P of two-word determinants: static
    heat-bath screening without ``psi``, dynamic amplitude screening with
    it."""
    d = _dets4(dets)
    n = d.shape[0]
    p = None
    if psi is not None:
        p = _f64(psi)
        if (p.shape[0] if isinstance(p, np.ndarray) else p.numel()) != n:
            raise ValueError("size mismatch: dets_V and psi_v")
    h = C.c_void_p()
    N.check(N.lib.dnq_wide_build(ctx.handle, N.ptr(d), n, N.ptr(p), int(n_orb), float(eps1),
                                 N.stream_of(d, p), C.byref(h)))
    H = DeviceHamiltonian(h.value)
    H.words = 2
    return H


def _blocks(H: DeviceHamiltonian) -> dict:
    return {"H_VV": H.to_coo(0), "H_VP": H.to_coo(1), "det_P": H.dets_p(), "size_P": H.n_p}


def get_ham_conn_wide(dets_V, int_ctx: IntCtx, n_orb: int, eps1: float = 1e-6) -> dict:
    """``get_ham_conn(use_heatbath=True)`` for two-word determinants."""
    H = build_wide(int_ctx, dets_V, n_orb=n_orb, eps1=eps1)
    try:
        return _blocks(H)
    finally:
        H.close()


def get_ham_conn_amp_wide(dets_V, psi_v, int_ctx: IntCtx, n_orb: int,
                          eps1: float = 1e-6) -> dict:
    """``get_ham_conn_amp`` for two-word determinants."""
    H = build_wide(int_ctx, dets_V, psi_v, n_orb=n_orb, eps1=eps1)
    try:
        return _blocks(H)
    finally:
        H.close()


def p_diag(H: DeviceHamiltonian, ctx: IntCtx, out=None):
    """diag(H_PP) of a (one- or two-word) handle, host or device output."""
    if out is None:
        out = np.empty(H.n_p, np.float64)
    N.check(N.lib.dnq_ham_p_diag(H._h, ctx.handle, N.ptr(out), N.stream_of(out)))
    return out


def ham_eff_wide(H: DeviceHamiltonian, h_pp, e_ref: float, *, reg_type: str = "sigma",
                 epsilon: float = 1e-12, precision: int = N.F64) -> DeviceHamiltonian:
    """H_eff = H_VV + H_VP (e_ref - H_PP)^-1 H_PV on the device
    (ham_eff.cpp:64-233), from a device-resident build."""
    if reg_type not in ("sigma", "linear_shift"):
        raise ValueError(f"invalid reg_type: {reg_type}")
    h = C.c_void_p()
    N.check(N.lib.dnq_ham_eff_from(H._h, N.ptr(h_pp), float(e_ref),
                                   1 if reg_type == "sigma" else 0, float(epsilon),
                                   int(precision), N.stream_of(h_pp), C.byref(h)))
    return DeviceHamiltonian(h.value)


__all__ = ["IntCtxWide", "get_ham_diag_wide", "build_wide", "get_ham_conn_wide",
           "get_ham_conn_amp_wide", "p_diag", "ham_eff_wide"]
