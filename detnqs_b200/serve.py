"""Device-resident serving loop.

A :class:`Server` keeps screened H_VV blocks of registered systems resident
on the GPU and answers build and local-energy requests from many clients.
Requests are admitted by free device memory (a byte budget with
least-recently-used eviction of idle blocks), builds run on several streams
at once, and local-energy requests that arrive while a grouped launch runs
are collected into the next one (continuous batching).  A request's result
does not depend on the requests served beside it.

The native runtime (scheduler, workers, admission) is ``dnq_server_*`` in
``libdetnqs_b200``; this module is its Python face.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import native as N

BUILD = N.REQ_BUILD
ELOC = N.REQ_ELOC


@dataclass
class Ticket:
    """A submitted request; holds the host buffers until it is waited on."""
    id: int
    kind: int
    sys: int
    psi: np.ndarray | None = None
    eloc: np.ndarray | None = None
    result: dict | None = field(default=None, repr=False)


class Server:
    def __init__(self, *, device: int = 0, budget_bytes: float = 150e9, build_slots: int = 2,
                 max_group: int = 64):
        h = C.c_void_p()
        N.check(N.lib.dnq_server_create(int(device), int(budget_bytes), int(build_slots),
                                        int(max_group), C.byref(h)))
        self._h = h
        self._keep = []            # contexts and determinant arrays of the systems
        self.sizes: list[int] = []

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.check(N.lib.dnq_server_destroy(self._h))
            self._h = C.c_void_p(None)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_system(self, ctx, dets, n_orb: int, *, policy: int = N.POLICY_STATIC,
                   use_heatbath: bool = True, eps1: float = 1e-7) -> int:
        """Register a system (integral context + determinant set); returns
        its id.  Nothing is built until a request needs it."""
        d = np.ascontiguousarray(dets, dtype=np.uint64)
        sid = C.c_int()
        N.check(N.lib.dnq_server_add_system(self._h, ctx.handle, d.ctypes.data, d.shape[0],
                                            int(n_orb), int(policy), int(bool(use_heatbath)),
                                            float(eps1), C.byref(sid)))
        self._keep.append((ctx, d))
        self.sizes.append(d.shape[0])
        return sid.value

    def submit(self, kind: int, sys: int, psi=None, *, want_eloc: bool = False,
               precision: int = N.F32) -> Ticket:
        p = None if psi is None else np.ascontiguousarray(psi, dtype=np.float64)
        e = np.empty(self.sizes[sys]) if (want_eloc and p is not None) else None
        rid = C.c_int64()
        N.check(N.lib.dnq_server_submit(self._h, int(kind), int(sys),
                                        None if p is None else p.ctypes.data,
                                        None if e is None else e.ctypes.data,
                                        int(precision), C.byref(rid)))
        return Ticket(rid.value, kind, sys, p, e)

    def wait(self, t: Ticket, timeout: float = 600.0) -> dict:
        """Result of a request: energy terms, latency and queueing time (s),
        nnz of a block it built, local energies if asked for."""
        if t.result is not None:
            return t.result
        out = np.zeros(4)
        nnz = C.c_int64()
        N.check(N.lib.dnq_server_wait(self._h, t.id, float(timeout), out.ctypes.data,
                                      C.byref(nnz)))
        num, den = float(out[0]), float(out[1])
        t.result = {"num": num, "den": den, "energy": num / den if den else None,
                    "latency_s": float(out[2]), "queue_s": float(out[3]), "nnz": nnz.value,
                    "eloc": t.eloc}
        return t.result

    def set_budget(self, budget_bytes: float):
        """New admission budget; idle blocks above it are evicted at once,
        least recently used first."""
        N.check(N.lib.dnq_server_set_budget(self._h, int(budget_bytes)))

    def pause(self, paused: bool = True):
        """Hold (or release) grouped local-energy launches; requests are
        still admitted and builds still run."""
        N.check(N.lib.dnq_server_pause(self._h, int(bool(paused))))

    def stats(self) -> dict:
        st = np.zeros(14)
        N.check(N.lib.dnq_server_stats(self._h, st.ctypes.data))
        keys = ("completed", "failed", "builds", "groups", "mean_group", "max_group",
                "evictions", "resident_bytes", "peak_bytes", "resident_blocks", "pending",
                "ready", "build_seconds", "group_seconds")
        return dict(zip(keys, (float(x) for x in st)))


__all__ = ["Server", "Ticket", "BUILD", "ELOC"]
