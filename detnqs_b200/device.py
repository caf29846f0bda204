"""Device-resident Hamiltonian blocks (a handle around ``dnq_ham_t``).

A :class:`DeviceHamiltonian` keeps H_VV (and H_VP / the P set when built) in
HBM in CSR form, so H.psi, local energies and the proxy operator run on the
GPU without copying the matrix back to the host.  ``to_coo`` / ``to_scipy``
produce the reference's host formats on request.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N


def _dets(x) -> np.ndarray:
    if hasattr(x, "is_cuda") and x.is_cuda:
        if x.ndim != 2 or x.shape[1] != 2:
            raise ValueError("determinants must have shape (N, 2)")
        return x.contiguous()
    a = np.ascontiguousarray(x, dtype=np.uint64)
    if a.ndim != 2 or a.shape[1] != 2:
        raise ValueError("determinants must be uint64[N, 2]")
    return a


def _f64(x, n: int | None = None):
    if hasattr(x, "is_cuda") and x.is_cuda:
        import torch
        t = x.to(torch.float64).contiguous()
        if n is not None and t.numel() != n:
            raise ValueError("size mismatch")
        return t
    a = np.ascontiguousarray(x, dtype=np.float64)
    if n is not None and a.shape[0] != n:
        raise ValueError("size mismatch")
    return a


def _f64_2d(X, n: int):
    """n x k FP64, C order (numpy or CUDA tensor)."""
    if hasattr(X, "is_cuda") and X.is_cuda:
        import torch
        t = X.to(torch.float64).contiguous()
        if t.dim() != 2 or t.shape[0] != n:
            raise ValueError("X must be n_V x k")
        return t
    a = np.ascontiguousarray(X, dtype=np.float64)
    if a.ndim != 2 or a.shape[0] != n:
        raise ValueError("X must be n_V x k")
    return a


class DeviceHamiltonian:
    """Owner of one ``dnq_ham_t``."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)
        info = np.zeros(6, np.int64)
        N.check(N.lib.dnq_ham_info(self._h, info.ctypes.data))
        self.n_v, self.nnz_vv, self.n_p, self.nnz_vp, self.candidates, self.device_bytes = (
            int(v) for v in info)

    # -- lifetime ------------------------------------------------------------
    def close(self) -> None:
        if self._h and self._h.value:
            N.check(N.lib.dnq_ham_destroy(self._h))
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def set_option(self, option: int, value: int) -> None:
        """H.psi shape of this handle alone (N.OPT_SPMV_LANES: 0/4/8/16/32
        lanes per row; N.OPT_SPMV_UNROLL: 0/1/2/4 slots per lane; 0 = by
        the average row length)."""
        N.check(N.lib.dnq_ham_set_option(self._h, option, int(value)))

    def timings(self) -> dict:
        """Device time (ms) of the build phases, from CUDA events."""
        t = np.zeros(8)
        N.check(N.lib.dnq_ham_timings(self._h, t.ctypes.data))
        keys = ("maps_diag", "count", "scan_alloc", "fill", "sort_v", "p_discovery", "total")
        return dict(zip(keys, (float(x) for x in t[:7])))

    # -- copies to the host ----------------------------------------------------
    def to_coo(self, block: int = 0) -> dict:
        nnz = self.nnz_vv if block == 0 else self.nnz_vp
        rows = np.empty(nnz, np.uint32)
        cols = np.empty(nnz, np.uint32)
        vals = np.empty(nnz, np.float64)
        N.check(N.lib.dnq_ham_copy_coo(self._h, block, rows.ctypes.data, cols.ctypes.data,
                                       vals.ctypes.data, None))
        shape = (self.n_v, self.n_v) if block == 0 else (self.n_v, self.n_p)
        return {"row": rows, "col": cols, "val": vals, "shape": shape}

    def to_csr_arrays(self, block: int = 0):
        nnz = self.nnz_vv if block == 0 else self.nnz_vp
        rp = np.empty(self.n_v + 1, np.int64)
        cols = np.empty(nnz, np.uint32)
        vals = np.empty(nnz, np.float64)
        N.check(N.lib.dnq_ham_copy_csr(self._h, block, rp.ctypes.data, cols.ctypes.data,
                                       vals.ctypes.data, None))
        return rp, cols, vals

    def to_scipy(self, block: int = 0):
        import scipy.sparse as sp
        rp, cols, vals = self.to_csr_arrays(block)
        shape = (self.n_v, self.n_v) if block == 0 else (self.n_v, self.n_p)
        return sp.csr_matrix((vals, cols.astype(np.int64), rp), shape=shape)

    words = 1   # uint64 words per spin string (2 for handles of the wide build)

    def dets_p(self) -> np.ndarray:
        out = np.empty((self.n_p, 2 * self.words), np.uint64)
        N.check(N.lib.dnq_ham_copy_dets_p(self._h, out.ctypes.data, None))
        return out

    def diagonal(self) -> np.ndarray:
        out = np.empty(self.n_v, np.float64)
        N.check(N.lib.dnq_ham_copy_diag(self._h, out.ctypes.data, None))
        return out

    # -- operators ---------------------------------------------------------------
    def spmv(self, x, out=None, precision: int = N.F64):
        """y = H_VV x; x, out may be numpy (host) or CUDA tensors."""
        x = _f64(x, self.n_v)
        if out is None:
            if isinstance(x, np.ndarray):
                out = np.empty(self.n_v, np.float64)
            else:
                import torch
                out = torch.empty(self.n_v, dtype=torch.float64, device=x.device)
        N.check(N.lib.dnq_ham_spmv(self._h, N.ptr(x), N.ptr(out), precision,
                                   N.stream_of(x, out)))
        return out

    def proxy_spmv(self, xv, xp, diag_p, precision: int = N.F64):
        xv = _f64(xv, self.n_v)
        xp = _f64(xp, self.n_p)
        dp = _f64(diag_p, self.n_p)
        on_host = isinstance(xv, np.ndarray)
        if on_host:
            yv = np.empty(self.n_v)
            yp = np.empty(self.n_p)
        else:
            import torch
            yv = torch.empty(self.n_v, dtype=torch.float64, device=xv.device)
            yp = torch.empty(self.n_p, dtype=torch.float64, device=xv.device)
        N.check(N.lib.dnq_ham_proxy_spmv(self._h, N.ptr(xv), N.ptr(xp), N.ptr(dp), N.ptr(yv),
                                         N.ptr(yp), precision, N.stream_of(xv, xp)))
        return yv, yp

    def spmv_multi(self, X, out=None, precision: int = N.F64):
        """Y = H_VV X for the k columns of X (n_V x k, C order): one pass over
        the CSR for up to 8 (FP32) or 4 (FP64) vectors.  X, out may be numpy
        (host) or CUDA tensors."""
        X = _f64_2d(X, self.n_v)
        k = X.shape[1]
        if out is None:
            if isinstance(X, np.ndarray):
                out = np.empty((self.n_v, k), np.float64)
            else:
                import torch
                out = torch.empty((self.n_v, k), dtype=torch.float64, device=X.device)
        N.check(N.lib.dnq_ham_spmv_multi(self._h, N.ptr(X), N.ptr(out), k, precision,
                                         N.stream_of(X, out)))
        return out

    def local_energy_multi(self, X, eloc=None, precision: int = N.F64) -> np.ndarray:
        """Returns out[k, 2] = (x_j.Hx_j, x_j.x_j) of the columns of X; fills
        ``eloc`` (n_V x k) when given."""
        X = _f64_2d(X, self.n_v)
        k = X.shape[1]
        out = np.zeros(2 * k)
        N.check(N.lib.dnq_ham_local_energy_multi(self._h, N.ptr(X), N.ptr(eloc),
                                                 out.ctypes.data, k, precision,
                                                 N.stream_of(X, eloc)))
        return out.reshape(k, 2)

    def local_energy(self, x, eloc=None, precision: int = N.F64):
        """Returns (x.Hx, x.x); fills ``eloc`` (y_i / x_i) when given."""
        x = _f64(x, self.n_v)
        out2 = np.zeros(2)
        N.check(N.lib.dnq_ham_local_energy(self._h, N.ptr(x), N.ptr(eloc), out2.ctypes.data,
                                           precision, N.stream_of(x, eloc)))
        return float(out2[0]), float(out2[1])


def build(ctx, dets_V, *, n_orb: int, policy: int, use_heatbath: bool = False,
          eps1: float = 1e-6, psi=None, dets_ext=None, want_vp: bool = True) -> DeviceHamiltonian:
    """Run ``dnq_build`` and return the device-resident blocks."""
    V = _dets(dets_V)
    n = V.shape[0]
    X = None if dets_ext is None else _dets(dets_ext)
    p = None
    if policy == N.POLICY_DYNAMIC:
        if psi is None:
            raise ValueError("size mismatch: dets_V and psi_v")
        p = _f64(psi)
        if (p.shape[0] if isinstance(p, np.ndarray) else p.numel()) != n:
            raise ValueError("size mismatch: dets_V and psi_v")
    h = C.c_void_p()
    N.check(N.lib.dnq_build(ctx.handle, N.ptr(V), n, N.ptr(X), 0 if X is None else X.shape[0],
                            N.ptr(p), int(n_orb), int(policy), int(bool(use_heatbath)),
                            float(eps1), int(bool(want_vp)), N.stream_of(V, X, p),
                            C.byref(h)))
    return DeviceHamiltonian(h.value)
