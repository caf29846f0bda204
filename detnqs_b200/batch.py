"""Batched engine: many systems of uneven size in one launch per phase.

A :class:`Batch` holds, for every system, its integral context and its
determinant space; one :meth:`Batch.step` rebuilds every screened H_VV
(same rules and bit-identical results as the single-system build), applies
H to the concatenated amplitudes and returns per-system Rayleigh quotients
and local energies.  With ``graph=True`` the whole step is replayed from a
captured CUDA graph.  :func:`autotune` picks the kernel tunables for a
workload and caches the choice by workload signature.
"""

from __future__ import annotations

import ctypes as C
import json
import os
import time
from dataclasses import dataclass

import numpy as np

from . import native as N
from . import synthetic as S


class Batch:
    def __init__(self, ctxs, dets_list, n_orbs, *, policy: int = N.POLICY_STATIC,
                 use_heatbath: bool = True, eps1: float = 1e-7, device: int = 0, stream=None):
        self.n_sys = len(ctxs)
        if not (len(dets_list) == len(n_orbs) == self.n_sys):
            raise ValueError("one determinant array and n_orb per context")
        self._dets = [np.ascontiguousarray(d, dtype=np.uint64) for d in dets_list]
        ptrs = (C.c_void_p * self.n_sys)(*[d.ctypes.data for d in self._dets])
        hs = (C.c_void_p * self.n_sys)(*[c.handle.value for c in ctxs])
        nd = np.array([len(d) for d in self._dets], np.int64)
        no = np.array(n_orbs, np.int32)
        h = C.c_void_p()
        N.check(N.lib.dnq_batch_create(self.n_sys, hs, ptrs, nd.ctypes.data, no.ctypes.data,
                                       int(policy), int(bool(use_heatbath)), float(eps1),
                                       int(device), stream, C.byref(h)))
        self._h = h
        self._ctxs = list(ctxs)            # keep contexts alive
        self.offsets = np.concatenate([[0], np.cumsum(nd)])
        info = np.zeros(4, np.int64)
        N.check(N.lib.dnq_batch_info(self._h, info.ctypes.data))
        self.total, self.nnz, self.device_bytes = int(info[1]), int(info[2]), int(info[3])

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.check(N.lib.dnq_batch_destroy(self._h))
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def config(self):
        """(arena chunk, part-C search threshold, H.psi lanes per row,
        H.psi slots per lane); 0 = automatic for the last two."""
        c = np.zeros(4, np.int64)
        N.check(N.lib.dnq_batch_get_config(self._h, c.ctypes.data))
        return tuple(int(x) for x in c)

    @config.setter
    def config(self, cfg):
        c = np.zeros(4, np.int64)
        c[:len(cfg)] = cfg
        N.check(N.lib.dnq_batch_set_config(self._h, c.ctypes.data))

    def step(self, psi, *, precision: int = N.F32, graph: bool = False, stream=None,
             eloc=None):
        """One batched step (rebuild every H_VV, then H.psi).  Returns
        (energies[n_sys, 2] = {psi.H psi, psi.psi}, device ms)."""
        return self._run(N.lib.dnq_batch_step, psi, precision, graph, stream, eloc)

    def apply(self, psi, *, precision: int = N.F32, graph: bool = False, stream=None,
              eloc=None):
        """H.psi and energies on the resident H_VV blocks (no rebuild)."""
        return self._run(N.lib.dnq_batch_apply, psi, precision, graph, stream, eloc)

    def apply_multi(self, X, *, precision: int = N.F32, stream=None, eloc=None):
        """k amplitude sets per system in one pass over the resident blocks:
        X is total x k (C order, numpy or CUDA tensor; column j = the
        concatenated psi_j).  Returns (energies[n_sys, k, 2], device ms);
        column j equals apply(X[:, j]) bit for bit."""
        if hasattr(X, "data_ptr"):
            import torch
            Xp = X.to(torch.float64).contiguous()
        else:
            Xp = np.ascontiguousarray(X, np.float64)
        if Xp.ndim != 2 or Xp.shape[0] != self.total:
            raise ValueError("X must be total x k")
        k = int(Xp.shape[1])
        e2 = np.zeros((self.n_sys, k, 2))
        ms = C.c_double()
        N.check(N.lib.dnq_batch_apply_multi(self._h, N.ptr(Xp), N.ptr(eloc), e2.ctypes.data, k,
                                            int(precision), stream, C.byref(ms)))
        return e2, ms.value

    def _run(self, fn, psi, precision, graph, stream, eloc):
        p = psi if hasattr(psi, "data_ptr") else np.ascontiguousarray(psi, np.float64)
        e2 = np.zeros((self.n_sys, 2))
        ms = C.c_double()
        if graph and stream is None:
            stream = _side_stream()
        N.check(fn(self._h, N.ptr(p), N.ptr(eloc), e2.ctypes.data, int(precision),
                   int(bool(graph)), stream, C.byref(ms)))
        return e2, ms.value

    def timings(self) -> dict:
        """Device ms of the phases of the last eager step."""
        t = np.zeros(4)
        N.check(N.lib.dnq_batch_timings(self._h, t.ctypes.data))
        return dict(zip(("diag", "build", "compact", "hpsi"), (float(x) for x in t)))

    def coo(self, k: int) -> dict:
        nnz = C.c_int64()
        N.check(N.lib.dnq_batch_copy_coo(self._h, k, None, None, None, C.byref(nnz)))
        r = np.empty(nnz.value, np.uint32)
        c = np.empty(nnz.value, np.uint32)
        v = np.empty(nnz.value, np.float64)
        N.check(N.lib.dnq_batch_copy_coo(self._h, k, r.ctypes.data, c.ctypes.data, v.ctypes.data,
                                         C.byref(nnz)))
        n = len(self._dets[k])
        return {"row": r, "col": c, "val": v, "shape": (n, n)}


_STREAM = None


def _side_stream():
    """A non-default stream for graph capture (the legacy stream cannot be
    captured)."""
    global _STREAM
    if _STREAM is None:
        import torch
        _STREAM = torch.cuda.Stream()
    return _STREAM.cuda_stream


# ---------------------------------------------------------------------------
# Autotuner
# ---------------------------------------------------------------------------

CHUNKS = (2048, 8192, 32768)
GROUPS = (512, 2048, 8192)
LANES = (4, 8, 16, 32)
SLOTS = (1, 2, 4)


def signature(batch: Batch) -> str:
    """Workload key: size class of the batch (rows, nnz per row)."""
    rows = batch.total
    per_row = batch.nnz / max(rows, 1)
    return f"sys{batch.n_sys}-rows{int(np.log2(max(rows, 1)))}-nnz{int(np.log2(max(per_row, 1)))}"


def _time(batch: Batch, psi, reps: int, precision: int, apply: bool = False) -> float:
    ts = []
    run = batch.apply if apply else batch.step
    for _ in range(reps):
        _, ms = run(psi, precision=precision)
        ts.append(ms)
    return float(np.median(ts))


def autotune(batch: Batch, psi, *, reps: int = 3, precision: int = N.F32,
             cache: str | None = None) -> dict:
    """Coordinate search: (chunk, group threshold) of the build timed on the
    full step with automatic H.psi shape, then (lanes per row, slots per
    lane) of H.psi timed on H.psi alone.  The winner is set on the batch
    and stored under the workload signature in ``cache`` (JSON) if given."""
    key = signature(batch)
    if cache and os.path.exists(cache):
        with open(cache) as f:
            table = json.load(f)
        if key in table:
            batch.config = table[key]["config"]
            return table[key]
    t0 = time.perf_counter()
    results = []
    best = None
    for ch in CHUNKS:
        for g in GROUPS:
            batch.config = (ch, g, 0, 0)
            t = _time(batch, psi, reps, precision)
            results.append(((ch, g, 0, 0), t))
            if best is None or t < best[1]:
                best = ((ch, g, 0, 0), t)
    ch, g = best[0][:2]
    batch.config = (ch, g, 0, 0)
    batch.step(psi, precision=precision)
    hbest = None
    for lanes in LANES:
        for slots in SLOTS:
            batch.config = (ch, g, lanes, slots)
            t = _time(batch, psi, reps, precision, apply=True)
            results.append(((ch, g, lanes, slots), t))
            if hbest is None or t < hbest[1]:
                hbest = ((ch, g, lanes, slots), t)
    batch.config = hbest[0]
    best = (hbest[0], _time(batch, psi, reps, precision))
    entry = {"config": list(best[0]), "ms": best[1], "hpsi_ms": hbest[1], "signature": key,
             "tried": [[list(c), t] for c, t in results],
             "tune_seconds": time.perf_counter() - t0}
    if cache:
        table = {}
        if os.path.exists(cache):
            with open(cache) as f:
                table = json.load(f)
        table[key] = entry
        os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
        with open(cache, "w") as f:
            json.dump(table, f, indent=1)
    return entry


# ---------------------------------------------------------------------------
# Workload: many synthetic systems of uneven size
# ---------------------------------------------------------------------------

@dataclass
class BatchSystem:
    sysm: S.SyntheticSystem
    dets: np.ndarray


def _sample(job):
    n, na, nd, sys_seed, det_seed, path = job
    if path and os.path.exists(path):
        return np.load(path)
    sysm = S.make_system(n, na, na, 2 * n, sys_seed)
    V = S.heat_bath_sample(sysm, nd, det_seed, max_level=3)
    if path:
        np.save(path, V)
    return V


def make_batch_workload(n_sys: int = 64, seed: int = 77, n_min: int = 10, n_max: int = 40,
                        dets_min: float = 1e3, dets_max: float = 2e5,
                        cache_dir: str | None = None, workers: int | None = None
                        ) -> list[BatchSystem]:
    """n_orb uniform in [n_min, n_max]; n_elec an even number in
    [0.4, 0.6] * 2 n_orb with n_alpha = n_beta; K = 2 n_orb Cholesky vectors;
    determinant counts log-uniform in [dets_min, dets_max], HF plus sampled
    excitations up to triples.

    The systems are sampled in ``workers`` spawned processes (default: one
    per core, at most ``n_sys``); every system has its own seeds, so the
    result does not depend on the worker count."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n_sys):
        n = int(rng.integers(n_min, n_max + 1))
        lo, hi = int(np.ceil(0.4 * n)), int(np.floor(0.6 * n))
        na = int(rng.integers(lo, hi + 1))               # n_elec = 2 na, even
        nd = int(np.exp(rng.uniform(np.log(dets_min), np.log(dets_max))))
        path = None
        if cache_dir:
            os.makedirs(cache_dir, exist_ok=True)
            path = os.path.join(cache_dir, f"batch_{seed}_{k}_{n}_{na}_{nd}.npy")
        jobs.append((n, na, nd, seed * 1000 + k, seed * 7919 + k, path))
    workers = min(n_sys, workers or os.cpu_count() or 1)
    if workers > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        # largest first, spawned (safe whatever the parent has initialised)
        order = sorted(range(n_sys), key=lambda k: -jobs[k][2])
        with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            got = dict(zip(order, ex.map(_sample, [jobs[k] for k in order])))
        dets = [got[k] for k in range(n_sys)]
    else:
        dets = [_sample(j) for j in jobs]
    return [BatchSystem(S.make_system(n, na, na, 2 * n, ss), V)
            for (n, na, _, ss, _, _), V in zip(jobs, dets)]


__all__ = ["Batch", "autotune", "signature", "make_batch_workload", "BatchSystem"]
