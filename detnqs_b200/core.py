"""Drop-in for ``detnqs.core`` on the determinant-space Hamiltonian path.

Same function names, argument names, defaults, return formats and error
types as the reference's nanobind module (``csrc/bridge/bridge.cpp:235-772``,
stubs ``detnqs/core.pyi:74-356``); every call runs on the GPU through
libdetnqs_b200.so.  Inputs are host arrays (as in the reference) or CUDA
tensors; outputs are host numpy arrays in the reference's formats:

* determinants: ``uint64[N, 2]`` (alpha, beta);
* COO blocks: ``{"row": uint32, "col": uint32, "val": float64,
  "shape": (r, c)}`` sorted by (row, col), unique, zeros dropped.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N
from .device import DeviceHamiltonian, _dets, _f64, build

HEATBATH_THRESH = 1e-15   # csrc/detnqs/hamiltonian/ham_utils.hpp:42


class IntCtx:
    """Integral context resident in HBM (``IntCtx``, bridge.cpp:108-128).

    ``IntCtx(fcidump_path, num_orb)`` reads an FCIDUMP like the reference;
    :meth:`from_arrays` takes packed arrays (reference layout) directly.
    """

    def __init__(self, fcidump_path: str, num_orb: int, device: int = 0):
        h = C.c_void_p()
        N.check(N.lib.dnq_ctx_create_fcidump(str(fcidump_path).encode(), int(num_orb),
                                             int(device), C.byref(h)))
        self._h = h
        self.n_orb = int(num_orb)
        self.device = int(device)

    @classmethod
    def from_arrays(cls, num_orb: int, h1e, eri, e_nuc: float, device: int = 0) -> "IntCtx":
        obj = cls.__new__(cls)
        h1 = np.ascontiguousarray(h1e, np.float64)
        er = np.ascontiguousarray(eri, np.float64)
        n1 = num_orb * (num_orb + 1) // 2
        if h1.size != n1 or er.size != n1 * (n1 + 1) // 2:
            raise ValueError("packed integral arrays have the wrong length")
        h = C.c_void_p()
        N.check(N.lib.dnq_ctx_create(int(num_orb), h1.ctypes.data, er.ctypes.data,
                                     float(e_nuc), int(device), C.byref(h)))
        obj._h = h
        obj.n_orb = int(num_orb)
        obj.device = int(device)
        return obj

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def get_e_nuc(self) -> float:
        v = C.c_double()
        N.check(N.lib.dnq_ctx_e_nuc(self._h, C.byref(v)))
        return v.value

    def hb_prepare(self, threshold: float = HEATBATH_THRESH) -> None:
        N.check(N.lib.dnq_hb_prepare(self._h, float(threshold)))

    def hb_clear(self) -> None:
        N.check(N.lib.dnq_hb_clear(self._h))

    def hb_row(self, i: int, j: int):
        """(a, b, w) of heat-bath row {i, j} (weights descending)."""
        n = C.c_int64()
        N.check(N.lib.dnq_hb_row(self._h, i, j, None, None, None, 0, C.byref(n)))
        a = np.empty(n.value, np.int32)
        b = np.empty(n.value, np.int32)
        w = np.empty(n.value, np.float64)
        N.check(N.lib.dnq_hb_row(self._h, i, j, a.ctypes.data, b.ctypes.data, w.ctypes.data,
                                 n.value, C.byref(n)))
        return a, b, w

    def device_bytes(self) -> int:
        v = C.c_int64()
        N.check(N.lib.dnq_ctx_device_bytes(self._h, C.byref(v)))
        return v.value

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            N.check(N.lib.dnq_ctx_destroy(self._h))
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ctx(int_ctx) -> IntCtx:
    if not isinstance(int_ctx, IntCtx):
        raise TypeError("int_ctx must be a detnqs_b200.core.IntCtx")
    return int_ctx


# ---------------------------------------------------------------------------
# Hamiltonian construction (bridge.cpp:450-629)
# ---------------------------------------------------------------------------

def get_ham_diag(dets, int_ctx) -> np.ndarray:
    """<x|H|x> for each determinant (build_ham.cpp:388-400)."""
    ctx = _ctx(int_ctx)
    d = _dets(dets)
    n = d.shape[0]
    out = np.empty(n, np.float64)
    N.check(N.lib.dnq_ham_diag(ctx.handle, N.ptr(d), n, out.ctypes.data, N.stream_of(d)))
    return out


def get_ham_elems(bra, ket, int_ctx) -> np.ndarray:
    """HamEval::compute_elem for paired rows of ``bra`` and ``ket``."""
    ctx = _ctx(int_ctx)
    b = _dets(bra)
    k = _dets(ket)
    if b.shape != k.shape:
        raise ValueError("bra and ket must have the same shape")
    out = np.empty(b.shape[0], np.float64)
    N.check(N.lib.dnq_ham_elems(ctx.handle, N.ptr(b), N.ptr(k), b.shape[0], out.ctypes.data,
                                N.stream_of(b, k)))
    return out


def excitations(bra, ket, device: int = 0):
    """(degree, phase) of analyze_excitation for paired rows."""
    b = _dets(bra)
    k = _dets(ket)
    n = b.shape[0]
    deg = np.empty(n, np.int32)
    ph = np.empty(n, np.float64)
    N.check(N.lib.dnq_excitations(N.ptr(b), N.ptr(k), n, deg.ctypes.data, ph.ctypes.data,
                                  int(device), N.stream_of(b, k)))
    return deg, ph


def prepare_det_batch(dets, ref, n_orb: int, n_alpha: int, n_beta: int, kmax: int = 0,
                      need_k: bool = False, need_phase: bool = False, need_hp: bool = False,
                      need_hp_pos: bool = False, device: int = 0) -> dict:
    """Features of a determinant batch for the neural models, as
    detnqs.core.prepare_det_batch (bridge.cpp:347-430): a dict with "occ"
    int32[B, n_e] and, as asked, "k" / "phase" int8[B], "holes" / "parts"
    int32[B, kmax], "hp_mask" bool[B, kmax], "holes_pos" / "parts_pos"
    int32[B, kmax].  need_hp implies need_k.  Host determinants give numpy
    arrays (in page-locked memory); CUDA-tensor determinants give CUDA
    tensors on their device, computed on torch's current stream with no host
    copy."""
    d = _dets(dets)
    r = np.ascontiguousarray(ref, dtype=np.uint64).reshape(-1)
    if r.shape != (2,):
        raise ValueError(f"ref must be (2,), got {r.shape}")
    need_k = bool(need_k or need_hp)
    B, ne = int(d.shape[0]), int(n_alpha) + int(n_beta)
    kdim = max(int(kmax), 0)
    on_dev = hasattr(d, "is_cuda") and d.is_cuda
    import torch
    if on_dev:
        dev = d.device
        device = dev.index if dev.index is not None else torch.cuda.current_device()

        def new(shape, dt):
            return torch.empty(shape, dtype=getattr(torch, dt), device=dev)
    else:
        def new(shape, dt):   # page-locked, so the copies back run at full speed
            return torch.empty(shape, dtype=getattr(torch, dt), pin_memory=True).numpy()
    out = {"occ": new((B, max(ne, 0)), "int32")}
    if need_k:
        out["k"] = new((B,), "int8")
    if need_phase:
        out["phase"] = new((B,), "int8")
    if need_hp:
        out["holes"] = new((B, kdim), "int32")
        out["parts"] = new((B, kdim), "int32")
        out["hp_mask"] = new((B, kdim), "bool")   # one byte, 0 or 1
        if need_hp_pos:
            out["holes_pos"] = new((B, kdim), "int32")
            out["parts_pos"] = new((B, kdim), "int32")
    flags = ((N.NEED_K if need_k else 0) | (N.NEED_PHASE if need_phase else 0) |
             (N.NEED_HP if need_hp else 0) | (N.NEED_HP_POS if need_hp_pos else 0))
    p = lambda key: N.ptr(out[key]) if key in out else None  # noqa: E731
    N.check(N.lib.dnq_prepare_det_batch(N.ptr(d), B, r.ctypes.data, int(n_orb), int(n_alpha),
                                        int(n_beta), int(kmax), flags, p("occ"), p("k"),
                                        p("phase"), p("holes"), p("parts"), p("hp_mask"),
                                        p("holes_pos"), p("parts_pos"), int(device),
                                        N.stream_of(d)))
    return out


def _blocks(H: DeviceHamiltonian, with_p: bool) -> dict:
    out = {"H_VV": H.to_coo(0), "H_VP": H.to_coo(1)}
    if with_p:
        out["det_P"] = H.dets_p()
        out["size_P"] = H.n_p
    return out


def get_ham_vv(dets_V, int_ctx, n_orb: int) -> dict:
    """H_VV by full singles/doubles enumeration (build_ham.cpp:402-422)."""
    H = build(_ctx(int_ctx), dets_V, n_orb=n_orb, policy=N.POLICY_KNOWN_SETS, want_vp=False)
    try:
        return H.to_coo(0)
    finally:
        H.close()


def get_ham_block(bra_dets, ket_dets=None, int_ctx=None, n_orb: int | None = None) -> dict:
    """H_VV and H_VP for explicit spaces (build_ham.cpp:424-460)."""
    if int_ctx is None or n_orb is None:
        raise TypeError("get_ham_block() requires int_ctx and n_orb")
    ctx = _ctx(int_ctx)
    H = build(ctx, bra_dets, n_orb=n_orb, policy=N.POLICY_KNOWN_SETS, dets_ext=ket_dets,
              want_vp=ket_dets is not None)
    try:
        out = {"H_VV": H.to_coo(0), "H_VP": H.to_coo(1)}
        if ket_dets is not None and H.n_p > 0:
            out["det_P"] = H.dets_p()
            out["size_P"] = H.n_p
        if ket_dets is None:
            out["H_VP"] = {"row": np.empty(0, np.uint32), "col": np.empty(0, np.uint32),
                           "val": np.empty(0, np.float64), "shape": (0, 0)}
        return out
    finally:
        H.close()


def get_ham_conn(dets_V, int_ctx, n_orb: int, use_heatbath: bool = False,
                 eps1: float = 1e-6) -> dict:
    """H_VV / H_VP with static heat-bath screening and P discovery
    (build_ham.cpp:462-495)."""
    H = build(_ctx(int_ctx), dets_V, n_orb=n_orb, policy=N.POLICY_STATIC,
              use_heatbath=use_heatbath, eps1=eps1, want_vp=True)
    try:
        return _blocks(H, True)
    finally:
        H.close()


def get_ham_conn_amp(dets_V, psi_v, int_ctx, n_orb: int, eps1: float = 1e-6) -> dict:
    """Amplitude-weighted dynamic screening (build_ham.cpp:497-535)."""
    ctx = _ctx(int_ctx)
    V = _dets(dets_V)
    p = _f64(psi_v)
    if (p.shape[0] if isinstance(p, np.ndarray) else p.numel()) != V.shape[0]:
        raise ValueError("size mismatch: dets_V and psi_v")
    H = build(ctx, V, n_orb=n_orb, policy=N.POLICY_DYNAMIC, use_heatbath=True, eps1=eps1,
              psi=p, want_vp=True)
    try:
        return _blocks(H, True)
    finally:
        H.close()


def _coo_arrays(d: dict):
    r = np.ascontiguousarray(d["row"], dtype=np.uint32)
    c = np.ascontiguousarray(d["col"], dtype=np.uint32)
    v = np.ascontiguousarray(d["val"], dtype=np.float64)
    if not (r.shape == c.shape == v.shape):
        raise ValueError("COO arrays must have equal length")
    return r, c, v


def get_ham_eff(H_VV: dict, H_VP: dict, h_pp_diag, e_ref: float,
                reg_type: str = "sigma", epsilon: float = 1e-12,
                upper_only: bool = True, *, precision: str = "fp64",
                device: int = 0) -> dict:
    """H_eff = H_VV + H_VP D^-1 H_PV (ham_eff.cpp:64-233).

    ``upper_only`` is accepted and ignored, as in the reference
    (ham_eff.hpp:41).  ``precision="fp32"`` keeps H_VP values in FP32 with
    compensated accumulation (D^-1 and the H_VV add stay FP64).
    """
    if reg_type not in ("sigma", "linear_shift"):
        raise ValueError(f"invalid reg_type: {reg_type}")
    vr, vc, vv = _coo_arrays(H_VV)
    pr, pc, pv = _coo_arrays(H_VP)
    hpp = np.ascontiguousarray(h_pp_diag, dtype=np.float64)
    sv = tuple(int(x) for x in H_VV.get("shape", (0, 0)))
    sp_ = tuple(int(x) for x in H_VP.get("shape", (0, 0)))
    n_p = hpp.shape[0]
    if n_p > 0 and sp_[1] != n_p:
        raise ValueError("H_VP columns != h_pp_diag size")
    n_v = sv[0] if sv[0] else sp_[0]
    if n_p > 0 and sp_[0] != n_v:
        raise ValueError("H_VP rows != H_VV rows")
    h = C.c_void_p()
    N.check(N.lib.dnq_ham_eff(vr.ctypes.data, vc.ctypes.data, vv.ctypes.data, vv.size, n_v,
                              pr.ctypes.data, pc.ctypes.data, pv.ctypes.data, pv.size, n_p,
                              hpp.ctypes.data, float(e_ref), 1 if reg_type == "sigma" else 0,
                              float(epsilon), N.F32 if precision == "fp32" else N.F64,
                              int(device), None, C.byref(h)))
    H = DeviceHamiltonian(h.value)
    try:
        out = H.to_coo(0)
        if n_p == 0:
            out["shape"] = sv
        return out
    finally:
        H.close()


# ---------------------------------------------------------------------------
# Determinant generation (bridge.cpp:265-341)
# ---------------------------------------------------------------------------

_MODES = {"none": 0, "static": 1, "dynamic": 2}


def _gen(int_ctx, dets, n_orb, psi, mode: int, eps1: float) -> np.ndarray:
    d = _dets(dets)
    p = None if psi is None else _f64(psi)
    h = C.c_void_p()
    ctx = None if int_ctx is None else _ctx(int_ctx)
    N.check(N.lib.dnq_gen_dets(None if ctx is None else ctx.handle, N.ptr(d), d.shape[0],
                               int(n_orb), N.ptr(p), mode, float(eps1),
                               0 if ctx is None else ctx.device, N.stream_of(d, p),
                               C.byref(h)))
    H = DeviceHamiltonian(h.value)
    try:
        return H.dets_p()
    finally:
        H.close()


def gen_connected_dets(ref_dets, n_orb: int, device: int = 0) -> np.ndarray:
    """All unique singles and doubles of the references, sorted
    (det_space.cpp:167-213 + canonicalize)."""
    d = _dets(ref_dets)
    h = C.c_void_p()
    N.check(N.lib.dnq_gen_dets(None, N.ptr(d), d.shape[0], int(n_orb), None, -1, 0.0,
                               int(device), N.stream_of(d), C.byref(h)))
    H = DeviceHamiltonian(h.value)
    try:
        return H.dets_p()
    finally:
        H.close()


def gen_perturbative_dets(ref_dets, n_orb: int, int_ctx=None, psi_v=None,
                          mode: str = "none", eps1: float = 1e-6) -> np.ndarray:
    """P = C \\ V with optional heat-bath screening (bridge.cpp:278-341)."""
    if mode not in _MODES:
        raise ValueError(f"invalid screen mode: {mode}")
    m = _MODES[mode]
    if m == 0:
        d = _dets(ref_dets)
        h = C.c_void_p()
        dev = 0 if int_ctx is None else _ctx(int_ctx).device
        N.check(N.lib.dnq_gen_dets(None, N.ptr(d), d.shape[0], int(n_orb), None, 0, 0.0, dev,
                                   N.stream_of(d), C.byref(h)))
        H = DeviceHamiltonian(h.value)
        try:
            return H.dets_p()
        finally:
            H.close()
    if int_ctx is None:
        raise TypeError("screened modes need int_ctx")
    if m == 2:
        if psi_v is None:
            raise TypeError("dynamic mode needs psi_v")
        p = _f64(psi_v)
        if (p.shape[0] if isinstance(p, np.ndarray) else p.numel()) != _dets(ref_dets).shape[0]:
            raise ValueError("psi_v size mismatch")
        return _gen(int_ctx, ref_dets, n_orb, p, 2, eps1)
    return _gen(int_ctx, ref_dets, n_orb, None, 1, eps1)


def get_local_connections(dets, int_ctx, n_orb: int, use_heatbath: bool = False,
                          eps1: float = 1e-6) -> dict:
    """CSR-like local connectivity (local_conn.cpp:96-142): ``offsets``
    int32[N+1], ``dets`` uint64[M, 2], ``values`` float64[M]."""
    ctx = _ctx(int_ctx)
    d = _dets(dets)
    h = C.c_void_p()
    N.check(N.lib.dnq_local_connections(ctx.handle, N.ptr(d), d.shape[0], int(n_orb),
                                        int(bool(use_heatbath)), float(eps1),
                                        N.stream_of(d), C.byref(h)))
    H = DeviceHamiltonian(h.value)
    try:
        m = H.n_p
        off = np.empty(d.shape[0] + 1, np.int32)
        kd = np.empty((m, 2), np.uint64)
        vals = np.empty(m, np.float64)
        N.check(N.lib.dnq_conn_copy(H.handle, off.ctypes.data, kd.ctypes.data,
                                    vals.ctypes.data, None))
        return {"offsets": off, "dets": kd, "values": vals}
    finally:
        H.close()


def compute_pt2(dets_V, coeffs_V, int_ctx, n_orb: int, e_ref: float,
                use_heatbath: bool = False, eps1: float = 1e-6) -> dict:
    """Decomposed EN-PT2 (local_conn.cpp:247-418)."""
    ctx = _ctx(int_ctx)
    d = _dets(dets_V)
    c = _f64(coeffs_V)
    if (c.shape[0] if isinstance(c, np.ndarray) else c.numel()) != d.shape[0]:
        raise ValueError("coefficient size mismatch")
    out = np.zeros(3)
    N.check(N.lib.dnq_pt2(ctx.handle, N.ptr(d), d.shape[0], N.ptr(c), int(n_orb),
                          float(e_ref), int(bool(use_heatbath)), float(eps1),
                          out.ctypes.data, N.stream_of(d, c)))
    return {"e_pt2_internal": float(out[0]), "e_pt2_external": float(out[1]),
            "n_ext": int(out[2])}


def compute_variational_energy(dets, coeffs, int_ctx, n_orb: int,
                               use_heatbath: bool = False, eps1: float = 1e-6) -> float:
    """<Psi|H|Psi> on a fixed basis, matrix-free (local_conn.cpp:148-229)."""
    ctx = _ctx(int_ctx)
    d = _dets(dets)
    c = _f64(coeffs)
    if (c.shape[0] if isinstance(c, np.ndarray) else c.numel()) != d.shape[0]:
        raise ValueError("coefficient size mismatch")
    out = C.c_double()
    N.check(N.lib.dnq_variational_energy(ctx.handle, N.ptr(d), d.shape[0], N.ptr(c),
                                         int(n_orb), int(bool(use_heatbath)), float(eps1),
                                         C.byref(out), N.stream_of(d, c)))
    return out.value


__all__ = [
    "IntCtx",
    "get_ham_diag",
    "get_ham_elems",
    "excitations",
    "prepare_det_batch",
    "get_ham_vv",
    "get_ham_block",
    "get_ham_conn",
    "get_ham_conn_amp",
    "get_ham_eff",
    "compute_variational_energy",
    "gen_connected_dets",
    "gen_perturbative_dets",
    "get_local_connections",
    "compute_pt2",
    "HEATBATH_THRESH",
]
