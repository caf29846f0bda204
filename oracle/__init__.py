"""CPU checkers for the determinant-space Hamiltonian path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import
this package.  The product library (``detnqs_b200``) never loads it.

Two interchangeable back ends implement the C interface in ``dq_api.h``:

* ``Checker.reference()`` -- the reference DetNQS C++ core compiled from its
  own sources (``oracle/_ref/libdetnqs_ref.so``, recipe ``oracle/Makefile``);
* ``Checker.port()``      -- ``oracle/oracle.cpp``, an independent restatement
  of the same algorithm (``oracle/liboracle.so``).

Both return results in the reference bridge's formats
(``csrc/bridge/bridge.cpp:173-196``): COO dicts with ``row``/``col`` uint32,
``val`` float64 and ``shape``; determinant arrays uint64[N, 2].
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libdetnqs_ref.so")
PORT_LIB = os.path.join(HERE, "liboracle.so")

_P = C.c_void_p
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C")


class OracleError(RuntimeError):
    pass


REFERENCE_ENV = "DETNQS_REFERENCE_ROOT"


def reference_root() -> str | None:
    """The reference source tree named by $DETNQS_REFERENCE_ROOT, if that
    variable is set and the tree is there."""
    root = os.environ.get(REFERENCE_ENV)
    return root if root and os.path.isdir(os.path.join(root, "csrc")) else None


def build(reference_root: str | None = None, quiet: bool = True) -> None:
    """Compile the restatement and, if a reference tree is given (or named
    by $DETNQS_REFERENCE_ROOT) and exists, the reference core.  Building the
    checker is not using it."""
    if reference_root is None:
        reference_root = globals()["reference_root"]()
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                   stdout=out, stderr=out)
    if reference_root and os.path.isdir(os.path.join(reference_root, "csrc")):
        subprocess.run(["make", "-C", HERE, "ref", f"REF={reference_root}"],
                       check=True, stdout=out, stderr=out)


def _bind(lib: C.CDLL) -> None:
    def f(name, res, *args):
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = list(args)
    f("dq_last_error", C.c_char_p)
    f("dq_ctx_from_fcidump", _P, C.c_char_p, C.c_int)
    f("dq_ctx_from_arrays", _P, C.c_int, _f64p, _f64p, C.c_double)
    f("dq_ctx_free", None, _P)
    f("dq_ctx_e_nuc", C.c_double, _P)
    f("dq_hb_prepare", C.c_int, _P, C.c_double)
    f("dq_hb_clear", C.c_int, _P)
    f("dq_hb_row", C.c_int64, _P, C.c_int, C.c_int, _i32p, _i32p, _f64p, C.c_int64)
    f("dq_analyze", C.c_int, _u64p, _u64p, C.POINTER(C.c_int), C.POINTER(C.c_double))
    f("dq_compute_elem", C.c_double, _P, _u64p, _u64p)
    f("dq_ham_diag", C.c_int, _P, _u64p, C.c_int64, _f64p)
    f("dq_get_ham_vv", _P, _P, _u64p, C.c_int64, C.c_int)
    f("dq_get_ham_block", _P, _P, _u64p, C.c_int64, _P, C.c_int64, C.c_int)
    f("dq_get_ham_conn", _P, _P, _u64p, C.c_int64, C.c_int, C.c_int, C.c_double)
    f("dq_get_ham_conn_amp", _P, _P, _u64p, C.c_int64, _f64p, C.c_int, C.c_double)
    f("dq_vv_hb_rows", _P, _P, _u64p, C.c_int64, C.c_int, C.c_double, _i64p, C.c_int64)
    f("dq_get_ham_eff", _P, _u32p, _u32p, _f64p, C.c_int64, C.c_uint32, C.c_uint32,
      _u32p, _u32p, _f64p, C.c_int64, C.c_uint32, C.c_uint32,
      _f64p, C.c_int64, C.c_double, C.c_int, C.c_double)
    f("dq_local_connections", _P, _P, _u64p, C.c_int64, C.c_int, C.c_int, C.c_double)
    f("dq_variational_energy", C.c_int, _P, _u64p, C.c_int64, _f64p, C.c_int, C.c_int,
      C.c_double, C.POINTER(C.c_double))
    f("dq_pt2", C.c_int, _P, _u64p, C.c_int64, _f64p, C.c_int, C.c_double, C.c_int,
      C.c_double, _f64p)
    f("dq_gen_connected", _P, _u64p, C.c_int64, C.c_int)
    f("dq_gen_perturbative", _P, _P, _u64p, C.c_int64, C.c_int, _P, C.c_int, C.c_double)
    f("dq_res_size", C.c_int64, _P, C.c_int)
    f("dq_res_coo", None, _P, C.c_int, _u32p, _u32p, _f64p, _u32p)
    f("dq_res_dets", None, _P, _u64p)
    f("dq_res_offsets", None, _P, _i32p)
    f("dq_res_values", None, _P, _f64p)
    f("dq_res_free", None, _P)
    f("dq_prepare_det_batch", C.c_int, _u64p, C.c_int64, _u64p, C.c_int, C.c_int, C.c_int,
      C.c_int, C.c_int, _i32p, _P, _P, _P, _P, _P, _P, _P)


def _dets(x) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.uint64)
    if a.ndim != 2 or a.shape[1] != 2:
        raise ValueError("determinants must be uint64[N, 2]")
    return a


class Checker:
    """One loaded checker library."""

    _cache: dict[str, C.CDLL] = {}

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise OracleError(f"checker library not built: {path}")
        if path not in Checker._cache:
            lib = C.CDLL(path)
            _bind(lib)
            Checker._cache[path] = lib
        self.lib = Checker._cache[path]
        self.path = path

    @classmethod
    def reference(cls) -> "Checker":
        return cls(REF_LIB)

    @classmethod
    def port(cls) -> "Checker":
        return cls(PORT_LIB)

    @staticmethod
    def reference_available() -> bool:
        return os.path.exists(REF_LIB)

    # -- helpers ------------------------------------------------------------
    def _err(self, what: str):
        raise OracleError(f"{what}: {self.lib.dq_last_error().decode()}")

    def _coo(self, r, which: int) -> dict:
        m = self.lib.dq_res_size(r, which)
        rows = np.empty(m, np.uint32)
        cols = np.empty(m, np.uint32)
        vals = np.empty(m, np.float64)
        shape = np.zeros(2, np.uint32)
        self.lib.dq_res_coo(r, which, rows, cols, vals, shape)
        return {"row": rows, "col": cols, "val": vals,
                "shape": (int(shape[0]), int(shape[1]))}

    def _dets_of(self, r) -> np.ndarray:
        m = self.lib.dq_res_size(r, 2)
        out = np.empty((m, 2), np.uint64)
        self.lib.dq_res_dets(r, out)
        return out

    def _take(self, r, what):
        if not r:
            self._err(what)
        return r

    # -- context ------------------------------------------------------------
    def ctx_from_fcidump(self, path: str, n_orb: int) -> "CheckerCtx":
        p = self.lib.dq_ctx_from_fcidump(path.encode(), n_orb)
        if not p:
            self._err("ctx_from_fcidump")
        return CheckerCtx(self, p, n_orb)

    def ctx_from_arrays(self, n_orb: int, h1e, eri, e_nuc: float) -> "CheckerCtx":
        p = self.lib.dq_ctx_from_arrays(n_orb, np.ascontiguousarray(h1e, np.float64),
                                        np.ascontiguousarray(eri, np.float64), e_nuc)
        if not p:
            self._err("ctx_from_arrays")
        return CheckerCtx(self, p, n_orb)

    def analyze(self, bra, ket) -> tuple[int, float]:
        d = C.c_int()
        ph = C.c_double()
        self.lib.dq_analyze(np.ascontiguousarray(bra, np.uint64),
                            np.ascontiguousarray(ket, np.uint64), C.byref(d), C.byref(ph))
        return d.value, ph.value

    def prepare_det_batch(self, dets, ref, n_orb: int, n_alpha: int, n_beta: int,
                          kmax: int = 0, need_k: bool = False, need_phase: bool = False,
                          need_hp: bool = False, need_hp_pos: bool = False) -> dict:
        """Features of a determinant batch, as the bridge's prepare_det_batch
        (bridge.cpp:347-430): a dict of occ and the fields asked for."""
        d = _dets(dets)
        r = np.ascontiguousarray(ref, np.uint64).reshape(2)
        B, ne = len(d), n_alpha + n_beta
        need_k = need_k or need_hp
        out = {"occ": np.zeros((B, max(ne, 0)), np.int32)}
        if need_k:
            out["k"] = np.zeros(B, np.int8)
        if need_phase:
            out["phase"] = np.zeros(B, np.int8)
        if need_hp:
            for key in ("holes", "parts", "holes_pos", "parts_pos")[:4 if need_hp_pos else 2]:
                out[key] = np.zeros((B, max(kmax, 0)), np.int32)
            out["hp_mask"] = np.zeros((B, max(kmax, 0)), np.uint8)
        ptr = lambda key: out[key].ctypes.data if key in out else None  # noqa: E731
        flags = (1 if need_k else 0) | (2 if need_phase else 0) | (4 if need_hp else 0) | \
                (8 if need_hp_pos else 0)
        rc = self.lib.dq_prepare_det_batch(d, B, r, n_orb, n_alpha, n_beta, kmax, flags,
                                           out["occ"], ptr("k"), ptr("phase"), ptr("holes"),
                                           ptr("parts"), ptr("hp_mask"), ptr("holes_pos"),
                                           ptr("parts_pos"))
        if rc != 0:
            raise ValueError(self.lib.dq_last_error().decode())
        if "hp_mask" in out:
            out["hp_mask"] = out["hp_mask"].astype(bool)
        return out

    def gen_connected_dets(self, ref_dets, n_orb: int) -> np.ndarray:
        d = _dets(ref_dets)
        r = self._take(self.lib.dq_gen_connected(d, len(d), n_orb), "gen_connected")
        try:
            return self._dets_of(r)
        finally:
            self.lib.dq_res_free(r)

    def get_ham_eff(self, H_VV: dict, H_VP: dict, h_pp_diag, e_ref: float,
                    reg_type: str = "sigma", epsilon: float = 1e-12) -> dict:
        if reg_type not in ("sigma", "linear_shift"):
            raise ValueError(f"invalid reg_type: {reg_type}")
        def arr(d):
            return (np.ascontiguousarray(d["row"], np.uint32),
                    np.ascontiguousarray(d["col"], np.uint32),
                    np.ascontiguousarray(d["val"], np.float64))
        vr, vc, vv = arr(H_VV)
        pr, pc, pv = arr(H_VP)
        hpp = np.ascontiguousarray(h_pp_diag, np.float64)
        sv = H_VV.get("shape", (0, 0))
        sp_ = H_VP.get("shape", (0, 0))
        r = self._take(self.lib.dq_get_ham_eff(
            vr, vc, vv, len(vv), sv[0], sv[1], pr, pc, pv, len(pv), sp_[0], sp_[1],
            hpp, len(hpp), float(e_ref), 1 if reg_type == "sigma" else 0,
            float(epsilon)), "get_ham_eff")
        try:
            return self._coo(r, 0)
        finally:
            self.lib.dq_res_free(r)


class CheckerCtx:
    """Integral context of one checker (mirrors the bridge's IntCtx)."""

    def __init__(self, chk: Checker, ptr, n_orb: int):
        self.chk = chk
        self.lib = chk.lib
        self.ptr = ptr
        self.n_orb = n_orb

    def __del__(self):
        try:
            if self.ptr:
                self.lib.dq_ctx_free(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def get_e_nuc(self) -> float:
        return self.lib.dq_ctx_e_nuc(self.ptr)

    def hb_prepare(self, threshold: float = 1e-15) -> None:
        if self.lib.dq_hb_prepare(self.ptr, threshold) != 0:
            self.chk._err("hb_prepare")

    def hb_clear(self) -> None:
        self.lib.dq_hb_clear(self.ptr)

    def hb_row(self, i: int, j: int):
        cap = 1 << 20
        a = np.empty(cap, np.int32)
        b = np.empty(cap, np.int32)
        w = np.empty(cap, np.float64)
        n = self.lib.dq_hb_row(self.ptr, i, j, a, b, w, cap)
        if n < 0:
            raise OracleError("heat-bath table not built")
        return a[:n].copy(), b[:n].copy(), w[:n].copy()

    def compute_elem(self, bra, ket) -> float:
        return self.lib.dq_compute_elem(self.ptr, np.ascontiguousarray(bra, np.uint64),
                                        np.ascontiguousarray(ket, np.uint64))

    def get_ham_diag(self, dets) -> np.ndarray:
        d = _dets(dets)
        out = np.empty(len(d))
        if self.lib.dq_ham_diag(self.ptr, d, len(d), out) != 0:
            self.chk._err("get_ham_diag")
        return out

    def _blocks(self, r, what, with_p=True) -> dict:
        r = self.chk._take(r, what)
        try:
            out = {"H_VV": self.chk._coo(r, 0), "H_VP": self.chk._coo(r, 1)}
            if with_p:
                P = self.chk._dets_of(r)
                out["det_P"] = P
                out["size_P"] = len(P)
            return out
        finally:
            self.lib.dq_res_free(r)

    def get_ham_vv(self, dets_V) -> dict:
        d = _dets(dets_V)
        r = self.chk._take(self.lib.dq_get_ham_vv(self.ptr, d, len(d), self.n_orb), "get_ham_vv")
        try:
            return self.chk._coo(r, 0)
        finally:
            self.lib.dq_res_free(r)

    def get_ham_block(self, bra_dets, ket_dets=None) -> dict:
        d = _dets(bra_dets)
        if ket_dets is None:
            r = self.lib.dq_get_ham_block(self.ptr, d, len(d), None, 0, self.n_orb)
            out = self._blocks(r, "get_ham_block", with_p=False)
            return out
        k = _dets(ket_dets)
        r = self.lib.dq_get_ham_block(self.ptr, d, len(d), k.ctypes.data, len(k), self.n_orb)
        out = self._blocks(r, "get_ham_block", with_p=True)
        if out["size_P"] == 0:
            del out["det_P"], out["size_P"]
        return out

    def get_ham_conn(self, dets_V, use_heatbath=False, eps1=1e-6) -> dict:
        d = _dets(dets_V)
        return self._blocks(self.lib.dq_get_ham_conn(self.ptr, d, len(d), self.n_orb,
                                                     int(use_heatbath), eps1), "get_ham_conn")

    def get_ham_conn_amp(self, dets_V, psi_v, eps1=1e-6) -> dict:
        d = _dets(dets_V)
        p = np.ascontiguousarray(psi_v, np.float64)
        if len(p) != len(d):
            raise ValueError("size mismatch: dets_V and psi_v")
        return self._blocks(self.lib.dq_get_ham_conn_amp(self.ptr, d, len(d), p, self.n_orb,
                                                         eps1), "get_ham_conn_amp")

    def vv_hb_rows(self, dets_V, rows, eps1) -> dict:
        d = _dets(dets_V)
        rr = np.ascontiguousarray(rows, np.int64)
        r = self.chk._take(self.lib.dq_vv_hb_rows(self.ptr, d, len(d), self.n_orb, eps1,
                                                  rr, len(rr)), "vv_hb_rows")
        try:
            return self.chk._coo(r, 0)
        finally:
            self.lib.dq_res_free(r)

    def get_local_connections(self, dets, use_heatbath=False, eps1=1e-6) -> dict:
        d = _dets(dets)
        r = self.chk._take(self.lib.dq_local_connections(self.ptr, d, len(d), self.n_orb,
                                                         int(use_heatbath), eps1),
                           "get_local_connections")
        try:
            n_off = self.lib.dq_res_size(r, 3)
            off = np.empty(n_off, np.int32)
            self.lib.dq_res_offsets(r, off)
            vals = np.empty(self.lib.dq_res_size(r, 4), np.float64)
            self.lib.dq_res_values(r, vals)
            return {"offsets": off, "dets": self.chk._dets_of(r), "values": vals}
        finally:
            self.lib.dq_res_free(r)

    def compute_variational_energy(self, dets, coeffs, use_heatbath=False, eps1=1e-6) -> float:
        d = _dets(dets)
        c = np.ascontiguousarray(coeffs, np.float64)
        out = C.c_double()
        if len(c) != len(d):
            raise ValueError("coefficient size mismatch")
        if self.lib.dq_variational_energy(self.ptr, d, len(d), c, self.n_orb,
                                          int(use_heatbath), eps1, C.byref(out)) != 0:
            self.chk._err("compute_variational_energy")
        return out.value

    def compute_pt2(self, dets_V, coeffs_V, e_ref, use_heatbath=False, eps1=1e-6) -> dict:
        d = _dets(dets_V)
        c = np.ascontiguousarray(coeffs_V, np.float64)
        out = np.zeros(3)
        if self.lib.dq_pt2(self.ptr, d, len(d), c, self.n_orb, float(e_ref),
                           int(use_heatbath), eps1, out) != 0:
            self.chk._err("compute_pt2")
        return {"e_pt2_internal": out[0], "e_pt2_external": out[1], "n_ext": int(out[2])}

    def gen_perturbative_dets(self, ref_dets, psi_v=None, mode="none", eps1=1e-6) -> np.ndarray:
        d = _dets(ref_dets)
        m = {"none": 0, "static": 1, "dynamic": 2}[mode]
        p = None
        if m == 2:
            pa = np.ascontiguousarray(psi_v, np.float64)
            p = pa.ctypes.data
        r = self.chk._take(self.lib.dq_gen_perturbative(self.ptr, d, len(d), self.n_orb, p, m,
                                                        eps1), "gen_perturbative_dets")
        try:
            return self.chk._dets_of(r)
        finally:
            self.lib.dq_res_free(r)


# ---------------------------------------------------------------------------
# Two-word determinants (up to 128 orbitals): oracle/wide.cpp
# ---------------------------------------------------------------------------

class WideChecker:
    """The restatement for W-word spin strings (W = 1 or 2), in
    ``oracle/liboracle.so``.  Determinants are uint64[N, 2W]: alpha words
    (low word first), then beta words."""

    def __init__(self, n_orb: int, h1e, eri, e_nuc: float):
        if not os.path.exists(PORT_LIB):
            raise OracleError(f"checker library not built: {PORT_LIB}")
        lib = Checker(PORT_LIB).lib
        if not getattr(lib, "_wide_bound", False):
            def f(name, res, *args):
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = list(args)
            f("dqw_ctx_from_arrays", _P, C.c_int, _f64p, _f64p, C.c_double)
            f("dqw_ctx_free", None, _P)
            f("dqw_hb_prepare", C.c_int, _P, C.c_double)
            f("dqw_diag", C.c_int, _P, C.c_int, _u64p, C.c_int64, _f64p)
            f("dqw_elem", C.c_double, _P, C.c_int, _u64p, _u64p)
            f("dqw_build", _P, _P, C.c_int, _u64p, C.c_int64, _P, C.c_int, C.c_double,
              C.c_int64, C.c_int64)
            lib._wide_bound = True
        self.lib = lib
        self.chk = Checker(PORT_LIB)
        self.n_orb = n_orb
        self.ptr = lib.dqw_ctx_from_arrays(n_orb, np.ascontiguousarray(h1e, np.float64),
                                           np.ascontiguousarray(eri, np.float64), e_nuc)
        if not self.ptr:
            raise OracleError(lib.dq_last_error().decode())

    def __del__(self):
        if getattr(self, "ptr", None):
            self.lib.dqw_ctx_free(self.ptr)
            self.ptr = None

    def hb_prepare(self, threshold: float = 1e-15):
        if self.lib.dqw_hb_prepare(self.ptr, threshold):
            raise OracleError(self.lib.dq_last_error().decode())

    @staticmethod
    def _words(d: np.ndarray) -> int:
        if d.ndim != 2 or d.shape[1] not in (2, 4):
            raise ValueError("determinants must be uint64[N, 2] or uint64[N, 4]")
        return d.shape[1] // 2

    def diag(self, dets) -> np.ndarray:
        d = np.ascontiguousarray(dets, np.uint64)
        out = np.empty(len(d))
        self.lib.dqw_diag(self.ptr, self._words(d), d, len(d), out)
        return out

    def elem(self, bra, ket) -> float:
        b = np.ascontiguousarray(bra, np.uint64).reshape(-1)
        k = np.ascontiguousarray(ket, np.uint64).reshape(-1)
        return self.lib.dqw_elem(self.ptr, len(b) // 2, b, k)

    def build(self, dets, psi=None, *, eps1: float, rows=None) -> dict:
        """Screened blocks of rows [r0, r1) of ``dets`` (all rows by
        default): static heat-bath policy without ``psi``, the dynamic
        amplitude policy with it.  Returns H_VV, H_VP (COO dicts), det_P
        (uint64[N_P, 2W], sorted) and size_P."""
        d = np.ascontiguousarray(dets, np.uint64)
        W = self._words(d)
        r0, r1 = (0, len(d)) if rows is None else rows
        p = None if psi is None else np.ascontiguousarray(psi, np.float64)
        r = self.lib.dqw_build(self.ptr, W, d, len(d), None if p is None else p.ctypes.data,
                               self.n_orb, float(eps1), int(r0), int(r1))
        if not r:
            raise OracleError(self.lib.dq_last_error().decode())
        try:
            vv = self.chk._coo(r, 0)
            vp = self.chk._coo(r, 1)
            m = self.lib.dq_res_size(r, 2) * 2 // (2 * W)
            P = np.empty((m, 2 * W), np.uint64)
            if m:
                self.lib.dq_res_dets(r, P)
            return {"H_VV": vv, "H_VP": vp, "det_P": P, "size_P": m}
        finally:
            self.lib.dq_res_free(r)

