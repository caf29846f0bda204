"""The bench's CPU-baseline sample stays bounded when the host is noisy.

The sample size comes from a probe: the reference core's rows on 1024
random rows, less the per-call map of V (timed on one row).  A map call that
host noise slows past the probe used to leave a per-row cost of ~0 and size
the sample to every row of the space (a 486 s baseline on a busy host).
These tests drive both sizing functions with a fake checker on a virtual
clock; nothing is executed on a GPU and nothing sleeps.
"""

from __future__ import annotations

import numpy as np
import pytest


class _Clock:
    def __init__(self):
        self.t = 0.0

    def perf_counter(self):
        return self.t


class _Ctx:
    """vv_hb_rows costs map_s + rows * row_s of virtual time; the first
    one-row call costs `noise` more (a descheduled host thread)."""

    def __init__(self, clock, map_s, row_s, noise):
        self.clock, self.map_s, self.row_s, self.noise = clock, map_s, row_s, noise
        self.calls = []

    def hb_prepare(self, eps):
        pass

    def vv_hb_rows(self, V, rows, eps):
        extra = 0.0
        if len(rows) == 1 and self.noise:
            extra, self.noise = self.noise, 0.0
        self.clock.t += self.map_s + len(rows) * self.row_s + extra
        self.calls.append(len(rows))
        return {"val": np.zeros(len(rows) * 200)}


@pytest.fixture
def fake(monkeypatch):
    import bench
    import oracle
    clock = _Clock()
    state = {}

    class _Chk:
        def ctx_from_arrays(self, n_orb, h1e, eri, e_core):
            return state["ctx"]

        def ctx_from_fcidump(self, path, n_orb):
            return state["ctx"]

    monkeypatch.setattr(bench, "time", clock)
    monkeypatch.setattr(oracle, "PORT_LIB", __file__)
    monkeypatch.setattr(oracle.Checker, "reference_available", staticmethod(lambda: False))
    monkeypatch.setattr(oracle.Checker, "port", classmethod(lambda cls: _Chk()))

    def make(map_s, row_s, noise):
        state["ctx"] = _Ctx(clock, map_s, row_s, noise)
        return state["ctx"]
    return bench, make


class _Sys:
    n_orb = 30
    h1e = eri = None
    e_core = 0.0


V = np.zeros((1_000_000, 2), np.uint64)


@pytest.mark.parametrize("noise", [0.0, 0.3, 5.0])
def test_sample_bounded_under_noise(fake, noise):
    bench, make = fake
    # 0.5 s map, 0.5 ms per row: 15 s of rows is ~29k rows
    ctx = make(0.5, 5e-4, noise)
    rate, rows, nnz, t, threads, kind = bench.cpu_reference_sample(_Sys(), V, 15.0)
    assert kind == "port"
    assert 64 <= rows <= 120_000          # never the whole space: at most 4x the target
    assert t <= 4 * 15.0 + 1.0
    assert rate == pytest.approx(nnz / t)
    assert rows == pytest.approx(29_000, rel=0.02)   # one slow map call is outvoted


@pytest.mark.parametrize("noise", [0.0, 0.3, 5.0])
def test_rows_bounded_under_noise(fake, noise):
    bench, make = fake
    make(0.5, 5e-4, noise)
    rate, rows, nnz, t, threads, kind = bench.cpu_reference_rows([(_Sys(), V, 1e-6)], 15.0)
    assert 1024 <= rows <= 120_000        # at most 4x the target in any case
    assert t <= 4 * 15.0
    assert rows == pytest.approx(30_000, rel=0.02)   # one slow map call is outvoted
