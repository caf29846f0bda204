"""Lowest eigenvalue of a device-resident operator block.

The reference solves for the lowest root of its projected Hamiltonians with
dense or SciPy routines on the host (``detnqs/analysis/metrics.py``).  Here
the block stays in HBM: :func:`symmetric_part` forms 0.5 (H + H^T) on the
device (the screened blocks of the dynamic policy, and H_eff built from
them, are not symmetric), and :func:`lowest_eigenvalue` runs Lanczos with
full re-orthogonalisation, each step one FP64 ``H.spmv`` of the library.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N
from .device import DeviceHamiltonian


def symmetric_part(H: DeviceHamiltonian, stream=None) -> DeviceHamiltonian:
    """0.5 (H + H^T) of the V block, as a new handle."""
    h = C.c_void_p()
    N.check(N.lib.dnq_ham_symmetrize(H._h, stream, C.byref(h)))
    return DeviceHamiltonian(h.value)


def lowest_eigenvalue(H: DeviceHamiltonian, *, max_iter: int = 400, tol: float = 1e-13,
                      seed: int = 0, device: int = 0) -> tuple[float, int]:
    """Lowest eigenvalue of a symmetric block and the Lanczos steps used.

    Lanczos with full (twice-applied) re-orthogonalisation in FP64 on the
    device; the tridiagonal problem is solved on the host every 10 steps and
    the iteration stops once the lowest Ritz value changes by less than
    ``tol`` relative."""
    import torch
    from scipy.linalg import eigvalsh_tridiagonal

    n = H.n_v
    dev = torch.device("cuda", device)
    m = min(max_iter, n)
    g = torch.Generator().manual_seed(seed)
    Q = torch.empty((m + 1, n), dtype=torch.float64, device=dev)
    v = torch.randn(n, generator=g, dtype=torch.float64).to(dev)
    Q[0] = v / v.norm()
    w = torch.empty(n, dtype=torch.float64, device=dev)
    alphas: list[float] = []
    betas: list[float] = []
    prev = None
    theta = None
    for k in range(m):
        H.spmv(Q[k], out=w, precision=N.F64)
        a = torch.dot(w, Q[k])
        w -= a * Q[k]
        if k > 0:
            w -= betas[-1] * Q[k - 1]
        B = Q[:k + 1]
        for _ in range(2):
            w -= B.T @ (B @ w)
        b = float(w.norm())
        alphas.append(float(a))
        done = b <= 1e-14 * max(1.0, abs(alphas[-1]))
        if done or (k + 1) % 10 == 0 or k + 1 == m:
            theta = float(eigvalsh_tridiagonal(np.array(alphas), np.array(betas),
                                               select="i", select_range=(0, 0))[0])
            if done or (prev is not None and abs(theta - prev) <= tol * max(1.0, abs(theta))):
                return theta, k + 1
            prev = theta
        betas.append(b)
        Q[k + 1] = w / b
    return theta, m


__all__ = ["symmetric_part", "lowest_eigenvalue"]
