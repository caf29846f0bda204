"""Drop-in for ``detnqs.operator.hamiltonian`` (reference
``detnqs/operator/hamiltonian.py``): the same builders, dataclasses and
call signatures, with every block resident in HBM.

``system`` needs ``int_ctx`` (a :class:`detnqs_b200.core.IntCtx`) and
``n_orb``; ``space`` needs ``V_dets``.  The returned ``ham_vv`` / ``ham_vp``
/ ``ham_pv`` are :class:`DeviceBlock` objects with the SciPy calls the
reference's consumers use (``shape``, ``nnz``, ``dot``, ``diagonal``,
``tocoo``, ``tocsr``, ``transpose``).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Literal, NamedTuple, Tuple

import numpy as np

from .. import native as N
from ..device import DeviceHamiltonian, build


class DiagonalInfo(NamedTuple):
    """Diagonal elements H_ii for variational and perturbative spaces."""
    V: np.ndarray
    P: np.ndarray


class DeviceBlock:
    """One block (0 = H_VV, 1 = H_VP, 2 = H_PV) of a device-resident build."""

    def __init__(self, ham: DeviceHamiltonian, block: int):
        self._ham = ham
        self.block = block
        nv, np_ = ham.n_v, ham.n_p
        self.shape = {0: (nv, nv), 1: (nv, np_), 2: (np_, nv)}[block]
        self.nnz = ham.nnz_vv if block == 0 else ham.nnz_vp

    @property
    def device_hamiltonian(self) -> DeviceHamiltonian:
        return self._ham

    def dot(self, x, precision: int = N.F64):
        if self.block == 0:
            return self._ham.spmv(x, precision=precision)
        from ..device import _f64
        x = _f64(x, self.shape[1])
        if isinstance(x, np.ndarray):
            out = np.empty(self.shape[0], np.float64)
        else:
            import torch
            out = torch.empty(self.shape[0], dtype=torch.float64, device=x.device)
        N.check(N.lib.dnq_ham_block_spmv(self._ham.handle, self.block, N.ptr(x), N.ptr(out),
                                         precision, N.stream_of(x, out)))
        return out

    __matmul__ = dot

    def diagonal(self) -> np.ndarray:
        if self.block != 0:
            raise ValueError("diagonal() is defined for H_VV only")
        return np.asarray(self.tocsr().diagonal(), np.float64)

    def tocsr(self):
        if self.block == 2:
            return self._ham.to_scipy(1).T.tocsr()
        return self._ham.to_scipy(self.block)

    def tocoo(self):
        return self.tocsr().tocoo()

    def transpose(self):
        if self.block == 0:
            return self
        return DeviceBlock(self._ham, 2 if self.block == 1 else 1)

    T = property(transpose)

    def conjugate(self):
        return self            # real Hamiltonian


@dataclass(eq=False)
class VVHamiltonian:
    """Hamiltonian restricted to V (hamiltonian.py:38-50)."""
    ham_vv: DeviceBlock
    diagonals: DiagonalInfo


@dataclass(eq=False)
class ProxyHamiltonian:
    """Proxy Hamiltonian on T = V + P with diag(H_PP) (hamiltonian.py:53-68)."""
    ham_vv: DeviceBlock
    ham_vp: DeviceBlock
    ham_pv: DeviceBlock
    diagonals: DiagonalInfo


def _diag_v(H: DeviceHamiltonian) -> np.ndarray:
    d = H.diagonal()
    return np.where(np.abs(d) > 1e-15, d, 0.0)   # entries dropped from the CSR read 0


def build_vv_hamiltonian(system, space) -> VVHamiltonian:
    """H_VV for a fixed V (hamiltonian.py:86-114)."""
    V = np.ascontiguousarray(space.V_dets, dtype=np.uint64)
    H = build(system.int_ctx, V, n_orb=system.n_orb, policy=N.POLICY_KNOWN_SETS,
              want_vp=False)
    return VVHamiltonian(ham_vv=DeviceBlock(H, 0),
                         diagonals=DiagonalInfo(V=_diag_v(H), P=np.zeros((0,), np.float64)))


def build_proxy_hamiltonian(
    system,
    space,
    *,
    screening: Literal["none", "static", "dynamic"] = "static",
    psi_v: np.ndarray | None = None,
    screen_eps: float = 1e-6,
    diag_shift: float = 0.0,
) -> Tuple[ProxyHamiltonian, np.ndarray]:
    """H_VV, H_VP and diag(H_PP) with optional screening (hamiltonian.py:117-212)."""
    from .. import core
    V = np.ascontiguousarray(space.V_dets, dtype=np.uint64)
    n_v = V.shape[0]
    ctx = system.int_ctx
    if screening == "none":
        P = core.gen_perturbative_dets(V, system.n_orb, mode="none")
        H = build(ctx, V, n_orb=system.n_orb, policy=N.POLICY_KNOWN_SETS, dets_ext=P,
                  want_vp=True)
    elif screening == "static":
        H = build(ctx, V, n_orb=system.n_orb, policy=N.POLICY_STATIC, use_heatbath=True,
                  eps1=screen_eps, want_vp=True)
    elif screening == "dynamic":
        if psi_v is None:
            raise ValueError("Dynamic screening requires psi_v amplitudes on V")
        p = np.ascontiguousarray(psi_v, dtype=np.float64)
        if p.shape[0] != n_v:
            raise ValueError(f"psi_v shape mismatch: {p.shape[0]} != n_V={n_v}")
        H = build(ctx, V, n_orb=system.n_orb, policy=N.POLICY_DYNAMIC, use_heatbath=True,
                  eps1=screen_eps, psi=p, want_vp=True)
    else:
        raise ValueError(f"Unknown screening mode: {screening!r}")
    P_dets = H.dets_p()
    if H.n_p > 0:
        dp = np.empty(H.n_p, np.float64)
        N.check(N.lib.dnq_ham_p_diag(H.handle, ctx.handle, dp.ctypes.data, None))
        dp = dp + float(diag_shift)
    else:
        dp = np.zeros((0,), np.float64)
    ham = ProxyHamiltonian(ham_vv=DeviceBlock(H, 0), ham_vp=DeviceBlock(H, 1),
                           ham_pv=DeviceBlock(H, 2),
                           diagonals=DiagonalInfo(V=_diag_v(H), P=dp))
    return ham, P_dets


def build_effective_hamiltonian(
    system,
    proxy_ham: ProxyHamiltonian,
    e_ref: float,
    *,
    reg_type: Literal["sigma", "linear_shift"] = "sigma",
    epsilon: float = 1e-12,
    upper_only: bool = True,
    precision: Literal["fp64", "fp32"] = "fp64",
) -> VVHamiltonian:
    """Loewdin downfolding H_eff = H_VV + H_VP (e_ref - diag H_PP)^-1 H_PV on
    the device (hamiltonian.py:215-281; ham_eff.cpp:64-233)."""
    if reg_type not in ("sigma", "linear_shift"):
        raise ValueError(f"invalid reg_type: {reg_type}")
    src = proxy_ham.ham_vv.device_hamiltonian
    hpp = np.ascontiguousarray(proxy_ham.diagonals.P, dtype=np.float64)
    h = C.c_void_p()
    N.check(N.lib.dnq_ham_eff_from(src.handle, hpp.ctypes.data if hpp.size else None,
                                   float(e_ref), 1 if reg_type == "sigma" else 0,
                                   float(epsilon), N.F32 if precision == "fp32" else N.F64,
                                   None, C.byref(h)))
    H = DeviceHamiltonian(h.value)
    return VVHamiltonian(ham_vv=DeviceBlock(H, 0),
                         diagonals=DiagonalInfo(V=np.asarray(H.to_scipy(0).diagonal()),
                                                P=np.zeros((0,), np.float64)))


__all__ = [
    "DiagonalInfo",
    "DeviceBlock",
    "VVHamiltonian",
    "ProxyHamiltonian",
    "build_vv_hamiltonian",
    "build_proxy_hamiltonian",
    "build_effective_hamiltonian",
]
