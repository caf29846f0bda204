"""Batched engine: every system's block equals its single-system build bit
for bit; per-system energies match; graph replay equals eager execution;
the autotuner's choice does not change results."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_coo_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def workload():
    from detnqs_b200 import batch as B
    from detnqs_b200 import core
    w = B.make_batch_workload(n_sys=7, seed=5, n_min=8, n_max=24, dets_min=300, dets_max=6000)
    ctxs = []
    for bs in w:
        c = core.IntCtx.from_arrays(bs.sysm.n_orb, bs.sysm.h1e, bs.sysm.eri, bs.sysm.e_core)
        c.hb_prepare(1e-15)
        ctxs.append(c)
    return w, ctxs


def test_blocks_match_single_builds(workload):
    from detnqs_b200 import batch as B
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    w, ctxs = workload
    bt = B.Batch(ctxs, [x.dets for x in w], [x.sysm.n_orb for x in w], eps1=1e-7)
    for k, (bs, c) in enumerate(zip(w, ctxs)):
        H = D.build(c, bs.dets, n_orb=bs.sysm.n_orb, policy=N.POLICY_STATIC,
                    use_heatbath=True, eps1=1e-7, want_vp=False)
        assert_coo_equal(bt.coo(k), H.to_coo(0))
        H.close()
    bt.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_energies_graph_and_eager(workload, prec):
    from detnqs_b200 import batch as B
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    from detnqs_b200 import synthetic as S
    P = N.F64 if prec == "f64" else N.F32
    w, ctxs = workload
    bt = B.Batch(ctxs, [x.dets for x in w], [x.sysm.n_orb for x in w], eps1=1e-7)
    psi = np.concatenate([S.normalized_psi(len(x.dets), 10 + k) for k, x in enumerate(w)])
    e_eager, _ = bt.step(psi, precision=P)
    e_graph1, _ = bt.step(psi, precision=P, graph=True)
    e_graph2, _ = bt.step(psi, precision=P, graph=True)
    np.testing.assert_array_equal(e_graph1, e_eager)
    np.testing.assert_array_equal(e_graph2, e_eager)
    for k, (bs, c) in enumerate(zip(w, ctxs)):
        H = D.build(c, bs.dets, n_orb=bs.sysm.n_orb, policy=N.POLICY_STATIC,
                    use_heatbath=True, eps1=1e-7, want_vp=False)
        x = psi[bt.offsets[k]:bt.offsets[k + 1]]
        num, den = H.local_energy(x, precision=P)
        tol = 1e-12 if prec == "f64" else 1e-6
        assert abs(e_eager[k, 0] / e_eager[k, 1] - num / den) < tol
        H.close()
    bt.close()


def test_autotune_keeps_results(workload, tmp_path):
    from detnqs_b200 import batch as B
    from detnqs_b200 import synthetic as S
    w, ctxs = workload
    bt = B.Batch(ctxs, [x.dets for x in w], [x.sysm.n_orb for x in w], eps1=1e-7)
    psi = np.concatenate([S.normalized_psi(len(x.dets), 3 + k) for k, x in enumerate(w)])
    before = [bt.coo(k) for k in range(bt.n_sys)]
    e0, _ = bt.step(psi)
    entry = B.autotune(bt, psi, reps=1, cache=str(tmp_path / "tune.json"))
    assert tuple(entry["config"]) == bt.config
    e1, _ = bt.step(psi, graph=True)
    for k in range(bt.n_sys):
        assert_coo_equal(bt.coo(k), before[k])
    np.testing.assert_allclose(e1[:, 0] / e1[:, 1], e0[:, 0] / e0[:, 1], rtol=0, atol=1e-10)
    again = B.autotune(bt, psi, cache=str(tmp_path / "tune.json"))   # cache hit
    assert again["config"] == entry["config"]
    bt.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_apply_on_resident_blocks(workload, prec):
    """H.psi without a rebuild: right after creation (FP32 split made on
    first use), equal to the full step on the same psi bit for bit, and a
    new psi gives the single-system energies."""
    from detnqs_b200 import batch as B
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    from detnqs_b200 import synthetic as S
    P = N.F64 if prec == "f64" else N.F32
    w, ctxs = workload
    bt = B.Batch(ctxs, [x.dets for x in w], [x.sysm.n_orb for x in w], eps1=1e-7)
    psi = np.concatenate([S.normalized_psi(len(x.dets), 40 + k) for k, x in enumerate(w)])
    e_fresh, _ = bt.apply(psi, precision=P)
    e_step, _ = bt.step(psi, precision=P)
    e_app, _ = bt.apply(psi, precision=P)
    e_app_g, _ = bt.apply(psi, precision=P, graph=True)
    np.testing.assert_array_equal(e_fresh, e_step)
    np.testing.assert_array_equal(e_app, e_step)
    np.testing.assert_array_equal(e_app_g, e_step)
    psi2 = np.concatenate([S.normalized_psi(len(x.dets), 90 + k) for k, x in enumerate(w)])
    eloc = np.empty(bt.total)
    e2, _ = bt.apply(psi2, precision=P, graph=True, eloc=eloc)
    for k, (bs, c) in enumerate(zip(w, ctxs)):
        H = D.build(c, bs.dets, n_orb=bs.sysm.n_orb, policy=N.POLICY_STATIC,
                    use_heatbath=True, eps1=1e-7, want_vp=False)
        x = psi2[bt.offsets[k]:bt.offsets[k + 1]]
        el = np.empty(len(x))
        num, den = H.local_energy(x, eloc=el, precision=P)
        tol = 1e-12 if prec == "f64" else 1e-6
        assert abs(e2[k, 0] / e2[k, 1] - num / den) < tol
        np.testing.assert_allclose(eloc[bt.offsets[k]:bt.offsets[k + 1]], el, rtol=1e-12 if
                                   prec == "f64" else 1e-5, atol=1e-9)
        H.close()
    t = bt.timings()
    assert set(t) == {"diag", "build", "compact", "hpsi"} and t["build"] > 0
    bt.close()


# ---------------------------------------------------------------------------
# Mixed widths: systems of at most and of more than 32 orbitals in one batch
# (the per-row scan word), with one system above 20000 determinants (arena
# chunks overflow, long rows inside the batch)
# ---------------------------------------------------------------------------

@pytest.fixture(scope="module")
def mixed_workload():
    from detnqs_b200 import batch as B
    from detnqs_b200 import core
    # n_orb = [36, 33, 40, 34, 26, 28], dets = [22500, 4708, 6306, 2290, 39901, 4037]
    w = B.make_batch_workload(n_sys=6, seed=5, n_min=26, n_max=40, dets_min=2000,
                              dets_max=40000)
    ctxs = []
    for bs in w:
        c = core.IntCtx.from_arrays(bs.sysm.n_orb, bs.sysm.h1e, bs.sysm.eri, bs.sysm.e_core)
        c.hb_prepare(1e-15)
        ctxs.append(c)
    yield w, ctxs
    for c in ctxs:
        c.close()


def test_mixed_width_batch_matches_single_builds_and_oracle(mixed_workload, port):
    from detnqs_b200 import batch as B
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    from detnqs_b200 import synthetic as S
    w, ctxs = mixed_workload
    n_orbs = [x.sysm.n_orb for x in w]
    sizes = [len(x.dets) for x in w]
    assert min(n_orbs) <= 32 < max(n_orbs)
    assert max(sizes) > 20000
    bt = B.Batch(ctxs, [x.dets for x in w], n_orbs, eps1=1e-7)
    blocks = [bt.coo(k) for k in range(bt.n_sys)]
    for k, (bs, c) in enumerate(zip(w, ctxs)):
        H = D.build(c, bs.dets, n_orb=bs.sysm.n_orb, policy=N.POLICY_STATIC,
                    use_heatbath=True, eps1=1e-7, want_vp=False)
        assert_coo_equal(blocks[k], H.to_coo(0))
        H.close()
    # the largest system of each width, row by row against the oracle:
    # 32 random rows and the 16 longest
    for k in (int(np.argmax([s if n <= 32 else -1 for n, s in zip(n_orbs, sizes)])),
              int(np.argmax([s if n > 32 else -1 for n, s in zip(n_orbs, sizes)]))):
        bs, blk = w[k], blocks[k]
        lens = np.bincount(blk["row"].astype(np.int64), minlength=sizes[k])
        rows = np.unique(np.concatenate([
            np.argsort(-lens, kind="stable")[:16],
            np.random.default_rng(k).choice(sizes[k], 32, replace=False)]))
        o = port.ctx_from_arrays(bs.sysm.n_orb, bs.sysm.h1e, bs.sysm.eri, bs.sysm.e_core)
        o.hb_prepare(1e-15)
        want = o.vv_hb_rows(bs.dets, rows, 1e-7)
        sel = np.isin(blk["row"], rows)
        got = {"row": blk["row"][sel], "col": blk["col"][sel], "val": blk["val"][sel],
               "shape": blk["shape"]}
        assert_coo_equal(got, want)
    # energies of one step against the single-system path
    psi = np.concatenate([S.normalized_psi(n, 60 + k) for k, n in enumerate(sizes)])
    e, _ = bt.step(psi, precision=N.F64, graph=True)
    for k, (bs, c) in enumerate(zip(w, ctxs)):
        H = D.build(c, bs.dets, n_orb=bs.sysm.n_orb, policy=N.POLICY_STATIC,
                    use_heatbath=True, eps1=1e-7, want_vp=False)
        num, den = H.local_energy(psi[bt.offsets[k]:bt.offsets[k + 1]])
        assert abs(e[k, 0] / e[k, 1] - num / den) < 1e-12
        H.close()
    bt.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_apply_multi_equals_apply_per_column(workload, prec):
    """Several amplitude sets per system in one pass: every column's
    energies and local energies equal a single-set apply bit for bit."""
    from detnqs_b200 import batch as B
    from detnqs_b200 import native as N
    P = N.F64 if prec == "f64" else N.F32
    w, ctxs = workload
    bt = B.Batch(ctxs, [x.dets for x in w], [x.sysm.n_orb for x in w], eps1=1e-7)
    k = 6
    X = np.random.default_rng(12).normal(size=(bt.total, k))
    eloc = np.empty((bt.total, k))
    e, _ = bt.apply_multi(X, precision=P, eloc=eloc)
    for j in range(k):
        el = np.empty(bt.total)
        ej, _ = bt.apply(X[:, j].copy(), precision=P, eloc=el)
        np.testing.assert_array_equal(e[:, j, :].view(np.uint64), ej.view(np.uint64))
        np.testing.assert_array_equal(eloc[:, j].view(np.uint64), el.view(np.uint64))
    bt.close()
