"""Serving loop: every result is the same served alone and in a mix of
concurrent requests (bit for bit), agrees with the direct API, survives
eviction under a small memory budget, and errors are reported per request."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def systems():
    from detnqs_b200 import batch as B
    from detnqs_b200 import core
    from detnqs_b200 import synthetic as S
    w = B.make_batch_workload(n_sys=5, seed=11, n_min=8, n_max=22, dets_min=300, dets_max=5000,
                              workers=1)
    fam = S.scan_family(14, 5, 5, 28, 3, points=6)
    Vf = S.heat_bath_sample(fam[0], 2000, 9, max_level=3)
    items = [(bs.sysm, bs.dets) for bs in w] + [(f, Vf) for f in fam]
    ctxs = []
    for sysm, _ in items:
        c = core.IntCtx.from_arrays(sysm.n_orb, sysm.h1e, sysm.eri, sysm.e_core)
        c.hb_prepare(1e-15)
        ctxs.append(c)
    return items, ctxs


def requests(items):
    from detnqs_b200 import native as N
    from detnqs_b200 import serve as V
    from detnqs_b200 import synthetic as S
    out = []
    for k, (_, dets) in enumerate(items):
        n = len(dets)
        out.append((V.ELOC, k, S.normalized_psi(n, 100 + k), N.F32))
        out.append((V.BUILD, k, None, N.F64))
        out.append((V.ELOC, k, S.normalized_psi(n, 200 + k), N.F64))
        out.append((V.BUILD, k, S.normalized_psi(n, 300 + k), N.F32))
    return out


def serve(items, ctxs, reqs, *, alone, budget=8e9, slots=3):
    from detnqs_b200 import serve as V
    with V.Server(budget_bytes=budget, build_slots=slots) as srv:
        ids = [srv.add_system(c, d, s.n_orb, eps1=1e-7) for (s, d), c in zip(items, ctxs)]
        res = []
        if alone:
            for kind, k, psi, prec in reqs:
                t = srv.submit(kind, ids[k], psi, want_eloc=psi is not None, precision=prec)
                res.append(srv.wait(t))
        else:
            ts = [srv.submit(kind, ids[k], psi, want_eloc=psi is not None, precision=prec)
                  for kind, k, psi, prec in reqs]
            res = [srv.wait(t) for t in ts]
        return res, srv.stats()


def assert_same(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x["num"] == y["num"] and x["den"] == y["den"]
        if x["eloc"] is not None:
            np.testing.assert_array_equal(x["eloc"], y["eloc"])


def test_alone_equals_mix(systems):
    items, ctxs = systems
    reqs = requests(items)
    alone, _ = serve(items, ctxs, reqs, alone=True)
    mix, st = serve(items, ctxs, reqs, alone=False)
    assert_same(alone, mix)
    assert st["failed"] == 0 and st["completed"] == len(reqs)


def test_burst_is_grouped_and_unchanged(systems):
    """Local-energy requests that collect while launches are held run as one
    grouped launch, with the results they get one by one."""
    import time
    from detnqs_b200 import native as N
    from detnqs_b200 import serve as V
    from detnqs_b200 import synthetic as S
    items, ctxs = systems
    burst = [(k, S.normalized_psi(len(d), 500 + k), prec) for k, (_, d) in enumerate(items)
             for prec in (N.F32, N.F64)]
    with V.Server(budget_bytes=8e9, build_slots=3) as srv:
        ids = [srv.add_system(c, d, s.n_orb, eps1=1e-7) for (s, d), c in zip(items, ctxs)]
        for k in ids:
            srv.wait(srv.submit(V.BUILD, k))
        one = [srv.wait(srv.submit(V.ELOC, ids[k], psi, want_eloc=True, precision=p))
               for k, psi, p in burst]
        srv.pause(True)
        ts = [srv.submit(V.ELOC, ids[k], psi, want_eloc=True, precision=p)
              for k, psi, p in burst]
        deadline = time.time() + 30
        while srv.stats()["ready"] < len(burst) and time.time() < deadline:
            time.sleep(0.01)
        srv.pause(False)
        grouped = [srv.wait(t) for t in ts]
        st = srv.stats()
    assert st["max_group"] == len(burst)
    assert_same(one, grouped)


def test_results_match_direct_api(systems):
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    items, ctxs = systems
    reqs = requests(items)
    mix, _ = serve(items, ctxs, reqs, alone=False)
    for (kind, k, psi, prec), r in zip(reqs, mix):
        if psi is None:
            continue
        sysm, dets = items[k]
        H = D.build(ctxs[k], dets, n_orb=sysm.n_orb, policy=N.POLICY_STATIC,
                    use_heatbath=True, eps1=1e-7, want_vp=False)
        el = np.empty(len(dets))
        num, den = H.local_energy(psi, eloc=el, precision=N.F64)
        e64 = num / den
        if prec == N.F64:
            assert abs(r["energy"] - e64) < 1e-12
            np.testing.assert_allclose(r["eloc"], el, rtol=1e-12, atol=1e-10)
        else:
            assert abs(r["energy"] - e64) <= 1e-6
        H.close()


def test_small_budget_evicts_and_keeps_results(systems):
    """With six same-size blocks resident (bond-scan points), shrink the
    budget to half of them: later requests evict idle blocks and rebuild,
    within the budget, and return what they returned before."""
    from detnqs_b200 import native as N
    from detnqs_b200 import serve as V
    from detnqs_b200 import synthetic as S
    items, ctxs = systems
    scan = [k for k in range(len(items)) if len(items[k][1]) == len(items[-1][1])][-6:]
    reqs = [(k, S.normalized_psi(len(items[k][1]), 700 + k)) for k in scan]
    with V.Server(budget_bytes=8e9, build_slots=2) as srv:
        ids = {k: srv.add_system(ctxs[k], items[k][1], items[k][0].n_orb, eps1=1e-7)
               for k in scan}
        ref = [srv.wait(srv.submit(V.ELOC, ids[k], psi, want_eloc=True, precision=N.F64))
               for k, psi in reqs]
        total = srv.stats()["resident_bytes"]
        # a rebuild reserves 1.5 x (28 B per entry + 64 B per row)
        need = max(1.5 * (28 * r["nnz"] + 64 * len(items[k][1])) for (k, _), r in zip(reqs, ref))
        budget = max(total / 2, 1.05 * need)
        assert budget < total
        srv.set_budget(budget)
        ts = [srv.submit(V.ELOC, ids[k], psi, want_eloc=True, precision=N.F64)
              for k, psi in reqs * 3]
        got = [srv.wait(t) for t in ts]
        st = srv.stats()
    assert st["evictions"] > 0 and st["failed"] == 0
    assert st["peak_bytes"] <= budget
    assert_same(ref * 3, got)


def test_errors_are_per_request(systems):
    from detnqs_b200 import native as N
    from detnqs_b200 import serve as V
    items, ctxs = systems
    sysm, dets = items[0]
    with V.Server(budget_bytes=1024, build_slots=1) as srv:
        k = srv.add_system(ctxs[0], dets, sysm.n_orb, eps1=1e-7)
        t = srv.submit(V.BUILD, k)
        with pytest.raises(N.DetnqsError) as e:
            srv.wait(t)
        assert e.value.code == N.ERR_BUDGET
        with pytest.raises(ValueError):
            srv.submit(V.ELOC, 7, np.ones(3))
        with pytest.raises(ValueError):
            srv.submit(V.ELOC, k, None)


def test_wait_times_out_and_request_stays_pending(systems):
    """dnq_server_wait returns DNQ_ERR_TIMEOUT while a request is held (the
    server is paused) and the request completes afterwards, unchanged."""
    from detnqs_b200 import native as N
    from detnqs_b200 import serve as V
    from detnqs_b200 import synthetic as S
    items, ctxs = systems
    (sysm, dets), ctx = items[0], ctxs[0]
    psi = S.normalized_psi(len(dets), 77)
    with V.Server(budget_bytes=8e9, build_slots=1) as srv:
        k = srv.add_system(ctx, dets, sysm.n_orb, eps1=1e-7)
        srv.wait(srv.submit(V.BUILD, k))
        first = srv.wait(srv.submit(V.ELOC, k, psi, want_eloc=True, precision=N.F64))
        srv.pause(True)
        t = srv.submit(V.ELOC, k, psi, want_eloc=True, precision=N.F64)
        with pytest.raises(N.DetnqsError) as e:
            srv.wait(t, timeout=0.01)
        assert e.value.code == N.ERR_TIMEOUT
        srv.pause(False)
        late = srv.wait(t)
        st = srv.stats()
    assert_same([first], [late])
    assert st["failed"] == 0
