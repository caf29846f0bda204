"""Drop-in for ``detnqs.operator.kernel``: H.psi operators.

The reference evaluates H.psi with SciPy CSR matvecs on the host inside
``jax.pure_callback`` (``detnqs/operator/kernel.py:48-145``).  Here the
operator runs on the GPU against the device-resident blocks.  psi may be a
numpy array (host round trip, as the reference) or a CUDA tensor (stays in
HBM).  Complex amplitudes are handled as two real products (H is real).

``precision`` selects FP64 values, or FP32 values with compensated FP32
accumulation and the FP64 diagonal term.
"""

from __future__ import annotations

from typing import Callable, NamedTuple

import numpy as np

from .. import native as N
from .hamiltonian import ProxyHamiltonian, VVHamiltonian


class VVContraction(NamedTuple):
    """H_VV @ psi_V."""
    V: object


class ProxyContraction(NamedTuple):
    """V: H_VV psi_V + H_VP psi_P ; P: H_PV psi_V + diag(H_PP) psi_P."""
    V: object
    P: object


def _dtype_name(d) -> str:
    if d is None:
        return "float64"
    try:
        return np.dtype(d).name
    except TypeError:
        return str(d).replace("torch.", "")


def _apply_real(fn, x):
    """fn on real vectors; complex x -> fn(Re x) + i fn(Im x)."""
    if isinstance(x, np.ndarray):
        if np.iscomplexobj(x):
            return fn(np.ascontiguousarray(x.real)) + 1j * fn(np.ascontiguousarray(x.imag))
        return fn(x)
    if x.is_complex():
        return fn(x.real.contiguous()) + 1j * fn(x.imag.contiguous())
    return fn(x)


def _cast(y, name: str):
    if isinstance(y, np.ndarray):
        return np.asarray(y, dtype=name)
    import torch
    return y.to(getattr(torch, name))


def build_vv_operator(ham: VVHamiltonian, *, jax_dtype=None,
                      precision: int = N.F64) -> Callable:
    """psi_V -> VVContraction(V = H_VV psi_V) (kernel.py:48-84)."""
    name = _dtype_name(jax_dtype)
    blk = ham.ham_vv

    def operator(psi_v):
        y = _apply_real(lambda v: blk.dot(v, precision=precision), psi_v)
        return VVContraction(V=_cast(y, name))

    return operator


def build_proxy_operator(ham: ProxyHamiltonian, *, jax_dtype=None,
                         precision: int = N.F64) -> Callable:
    """(psi_V, psi_P) -> ProxyContraction (kernel.py:87-145)."""
    name = _dtype_name(jax_dtype)
    H = ham.ham_vv.device_hamiltonian
    dp = np.ascontiguousarray(ham.diagonals.P, dtype=np.float64)

    def real_pair(xv, xp):
        if isinstance(xv, np.ndarray):
            return H.proxy_spmv(xv, xp, dp, precision=precision)
        import torch
        d = torch.from_numpy(dp).to(xv.device)
        return H.proxy_spmv(xv, xp, d, precision=precision)

    def operator(psi_v, psi_p):
        cplx = (np.iscomplexobj(psi_v) if isinstance(psi_v, np.ndarray) else psi_v.is_complex())
        if cplx:
            yr = real_pair(psi_v.real, psi_p.real)
            yi = real_pair(psi_v.imag, psi_p.imag)
            yv, yp = yr[0] + 1j * yi[0], yr[1] + 1j * yi[1]
        else:
            yv, yp = real_pair(psi_v, psi_p)
        return ProxyContraction(V=_cast(yv, name), P=_cast(yp, name))

    return operator


def local_energy(ham: VVHamiltonian, psi_v, *, precision: int = N.F64):
    """(E, E_loc) with E = <psi|H|psi>/<psi|psi> and E_loc = (H psi)_i / psi_i."""
    H = ham.ham_vv.device_hamiltonian
    if isinstance(psi_v, np.ndarray):
        eloc = np.empty(H.n_v)
    else:
        import torch
        eloc = torch.empty(H.n_v, dtype=torch.float64, device=psi_v.device)
    num, den = H.local_energy(psi_v, eloc=eloc, precision=precision)
    return num / den, eloc


__all__ = [
    "VVContraction",
    "ProxyContraction",
    "build_vv_operator",
    "build_proxy_operator",
    "local_energy",
]
