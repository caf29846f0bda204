"""ctypes binding of libdetnqs_b200.so (declared in include/detnqs_gpu.h).

The library is built in-tree (``detnqs_b200/_lib``) by
``make -C detnqs_b200/csrc``.  Importing this module loads it; a missing
library is an ImportError -- there is no CPU fallback for any entry point.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libdetnqs_b200.so")

OK = 0
ERR_INVALID = 1
ERR_NO_HEATBATH = 2
ERR_DUPLICATE = 3
ERR_OUT_OF_MEMORY = 4
ERR_BUDGET = 5
ERR_OVERFLOW = 6
ERR_TIMEOUT = 7
ERR_CUDA = 8
ERR_IO = 9
ERR_RANGE = 10

POLICY_KNOWN_SETS = 0
POLICY_STATIC = 1
POLICY_DYNAMIC = 2
F64 = 0
F32 = 1
OPT_FORCE_WALK = 1
OPT_ARENA_CHUNK = 2
OPT_ARENA_CAP = 3
OPT_SPMV_LANES = 4
OPT_SPMV_UNROLL = 5
OPT_PARTC_GROUPWALK = 7
OPT_BUILD_F32 = 8
NEED_K, NEED_PHASE, NEED_HP, NEED_HP_POS = 1, 2, 4, 8
REQ_BUILD = 0
REQ_ELOC = 1

# Every symbol the header declares; tests check the library exports them.
EXPORTS = (
    "dnq_last_error", "dnq_version", "dnq_launch_count",
    "dnq_ctx_create", "dnq_ctx_create_fcidump", "dnq_ctx_destroy", "dnq_ctx_e_nuc",
    "dnq_ctx_device_bytes", "dnq_hb_prepare", "dnq_hb_clear", "dnq_hb_row",
    "dnq_ham_diag", "dnq_ham_elems", "dnq_excitations", "dnq_prepare_det_batch",
    "dnq_slogdet", "dnq_slogdet_grad",
    "dnq_build", "dnq_set_option", "dnq_ham_destroy", "dnq_ham_info", "dnq_ham_timings", "dnq_ham_copy_coo",
    "dnq_ham_copy_csr", "dnq_ham_copy_dets_p", "dnq_ham_copy_diag",
    "dnq_ham_spmv", "dnq_ham_proxy_spmv", "dnq_ham_local_energy",
    "dnq_variational_energy", "dnq_ham_eff", "dnq_ham_eff_from", "dnq_ham_p_diag",
    "dnq_ham_block_spmv", "dnq_gen_dets", "dnq_local_connections", "dnq_conn_copy",
    "dnq_pt2", "dnq_ham_local_energy_noalloc", "dnq_ham_spmv_multi",
    "dnq_ham_local_energy_multi",
    "dnq_batch_create", "dnq_batch_destroy", "dnq_batch_info", "dnq_batch_set_config",
    "dnq_batch_get_config", "dnq_batch_step", "dnq_batch_apply", "dnq_batch_timings", "dnq_batch_copy_coo",
    "dnq_batch_apply_multi", "dnq_sort_order", "dnq_ham_set_option",
    "dnq_server_create", "dnq_server_destroy", "dnq_server_add_system", "dnq_server_submit",
    "dnq_server_wait", "dnq_server_set_budget", "dnq_server_pause", "dnq_server_stats",
    "dnq_ctx_create_wide", "dnq_wide_diag", "dnq_wide_build", "dnq_ham_symmetrize",
)


class DetnqsError(RuntimeError):
    """A libdetnqs_b200 call failed (non-argument errors)."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libdetnqs_b200.so not built at {LIB_PATH}; run "
            "`make -C detnqs_b200/csrc` (nvcc, sm_100a)")
    return C.CDLL(LIB_PATH)


lib = _load()

_P = C.c_void_p
_I64 = C.c_int64
_D = C.c_double
_I = C.c_int


def _sig(name, *args):
    fn = getattr(lib, name)
    fn.restype = C.c_int
    fn.argtypes = list(args)


lib.dnq_last_error.restype = C.c_char_p
lib.dnq_last_error.argtypes = []
lib.dnq_version.restype = C.c_int
lib.dnq_launch_count.restype = C.c_int64
lib.dnq_launch_count.argtypes = []
_sig("dnq_ctx_create", _I, _P, _P, _D, _I, C.POINTER(_P))
_sig("dnq_ctx_create_fcidump", C.c_char_p, _I, _I, C.POINTER(_P))
_sig("dnq_ctx_destroy", _P)
_sig("dnq_ctx_e_nuc", _P, C.POINTER(_D))
_sig("dnq_ctx_device_bytes", _P, C.POINTER(_I64))
_sig("dnq_hb_prepare", _P, _D)
_sig("dnq_hb_clear", _P)
_sig("dnq_hb_row", _P, _I, _I, _P, _P, _P, _I64, C.POINTER(_I64))
_sig("dnq_ham_diag", _P, _P, _I64, _P, _P)
_sig("dnq_ham_elems", _P, _P, _P, _I64, _P, _P)
_sig("dnq_excitations", _P, _P, _I64, _P, _P, _I, _P)
_sig("dnq_slogdet", _P, _I64, _I, _I, _P, _P, _I, _P)
_sig("dnq_slogdet_grad", _P, _P, _I64, _I, _I, _P, _I, _P)
_sig("dnq_prepare_det_batch", _P, _I64, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P,
     _I, _P)
_sig("dnq_build", _P, _P, _I64, _P, _I64, _P, _I, _I, _I, _D, _I, _P, C.POINTER(_P))
_sig("dnq_ham_destroy", _P)
_sig("dnq_set_option", _I, _I64)
_sig("dnq_ham_set_option", _P, _I, _I64)
_sig("dnq_ham_info", _P, _P)
_sig("dnq_ham_timings", _P, _P)
_sig("dnq_ham_copy_coo", _P, _I, _P, _P, _P, _P)
_sig("dnq_ham_copy_csr", _P, _I, _P, _P, _P, _P)
_sig("dnq_ham_copy_dets_p", _P, _P, _P)
_sig("dnq_ham_copy_diag", _P, _P, _P)
_sig("dnq_ham_spmv", _P, _P, _P, _I, _P)
_sig("dnq_ham_proxy_spmv", _P, _P, _P, _P, _P, _P, _I, _P)
_sig("dnq_ham_local_energy", _P, _P, _P, _P, _I, _P)
_sig("dnq_ham_block_spmv", _P, _I, _P, _P, _I, _P)
_sig("dnq_ham_local_energy_noalloc", _P, _P, _P, _P, _I, _P)
_sig("dnq_ham_spmv_multi", _P, _P, _P, _I, _I, _P)
_sig("dnq_ham_local_energy_multi", _P, _P, _P, _P, _I, _I, _P)
_sig("dnq_ham_p_diag", _P, _P, _P, _P)
_sig("dnq_gen_dets", _P, _P, _I64, _I, _P, _I, _D, _I, _P, C.POINTER(_P))
_sig("dnq_local_connections", _P, _P, _I64, _I, _I, _D, _P, C.POINTER(_P))
_sig("dnq_conn_copy", _P, _P, _P, _P, _P)
_sig("dnq_pt2", _P, _P, _I64, _P, _I, _D, _I, _D, _P, _P)
_sig("dnq_batch_create", _I, _P, _P, _P, _P, _I, _I, _D, _I, _P, C.POINTER(_P))
_sig("dnq_batch_destroy", _P)
_sig("dnq_batch_info", _P, _P)
_sig("dnq_batch_set_config", _P, _P)
_sig("dnq_batch_get_config", _P, _P)
_sig("dnq_batch_step", _P, _P, _P, _P, _I, _I, _P, C.POINTER(_D))
_sig("dnq_batch_apply", _P, _P, _P, _P, _I, _I, _P, C.POINTER(_D))
_sig("dnq_batch_apply_multi", _P, _P, _P, _P, _I, _I, _P, C.POINTER(_D))
_sig("dnq_sort_order", _P, _I64, _I, _P, _P, _I, _P)
_sig("dnq_batch_timings", _P, _P)
_sig("dnq_batch_copy_coo", _P, _I, _P, _P, _P, C.POINTER(_I64))
_sig("dnq_server_create", _I, _I64, _I, _I, C.POINTER(_P))
_sig("dnq_server_destroy", _P)
_sig("dnq_server_add_system", _P, _P, _P, _I64, _I, _I, _I, _D, C.POINTER(_I))
_sig("dnq_server_submit", _P, _I, _I, _P, _P, _I, C.POINTER(_I64))
_sig("dnq_server_wait", _P, _I64, _D, _P, C.POINTER(_I64))
_sig("dnq_server_set_budget", _P, _I64)
_sig("dnq_server_pause", _P, _I)
_sig("dnq_server_stats", _P, _P)
_sig("dnq_ctx_create_wide", _I, _P, _P, _D, _I, C.POINTER(_P))
_sig("dnq_wide_diag", _P, _P, _I64, _P, _P)
_sig("dnq_wide_build", _P, _P, _I64, _P, _I, _D, _P, C.POINTER(_P))
_sig("dnq_ham_symmetrize", _P, _P, C.POINTER(_P))
_sig("dnq_ham_eff_from", _P, _P, _D, _I, _D, _I, _P, C.POINTER(_P))
_sig("dnq_variational_energy", _P, _P, _I64, _P, _I, _I, _D, C.POINTER(_D), _P)
_sig("dnq_ham_eff", _P, _P, _P, _I64, _I64, _P, _P, _P, _I64, _I64, _P, _D, _I, _D, _I, _I,
     _P, C.POINTER(_P))


def check(code: int) -> None:
    """Raise the Python exception the reference bridge would raise."""
    if code == OK:
        return
    msg = lib.dnq_last_error().decode(errors="replace")
    if code in (ERR_INVALID, ERR_NO_HEATBATH, ERR_DUPLICATE):
        raise ValueError(msg)          # std::invalid_argument under nanobind
    if code == ERR_RANGE:
        raise IndexError(msg)          # std::out_of_range
    if code == ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise DetnqsError(code, msg)


def ptr(a) -> int | None:
    """Address of a numpy array or torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(f"unsupported buffer type {type(a)!r}")


def stream_of(*arrays) -> int | None:
    """cudaStream_t to use: torch's current stream if any argument is a
    CUDA tensor, else the default stream."""
    for a in arrays:
        if hasattr(a, "is_cuda") and a.is_cuda:
            import torch
            return torch.cuda.current_stream(a.device).cuda_stream
    return None
