"""Determinant batch features (the reference's prepare_det_batch,
det_batch.cpp:184-318 via bridge.cpp:347-430).

CPU tests pin the oracle restatement to the reference's outputs in
tests/golden/det_batch.npz (made by tests/golden/make_det_batch.py) and, when
the reference core is compiled here, to the reference on fresh batches.  GPU
tests compare the CUDA kernel, through the C ABI, with the same fixture and
with the oracle on larger batches, device-resident batches included.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN

FLAGS = [(False, False, False, False), (True, True, False, False),
         (False, True, True, False), (True, True, True, True)]
ERROR_CASES = [
    dict(dets=[[7, 7]], ref=[7, 7], n_orb=65, n_alpha=3, n_beta=3),
    dict(dets=[[7, 7]], ref=[7, 7], n_orb=4, n_alpha=3, n_beta=3, kmax=2, need_hp_pos=True),
    dict(dets=[[7, 7]], ref=[7, 7], n_orb=4, n_alpha=3, n_beta=3, kmax=-1, need_hp=True),
    dict(dets=[[7, 7]], ref=[7, 7], n_orb=2, n_alpha=3, n_beta=3),
    dict(dets=[[7, 7]], ref=[7, 7], n_orb=4, n_alpha=2, n_beta=3),
    dict(dets=[[7, 7]], ref=[3, 7], n_orb=4, n_alpha=3, n_beta=3, need_phase=True),
    dict(dets=[[7, 7]], ref=[3, 7], n_orb=4, n_alpha=3, n_beta=3, kmax=2, need_hp=True,
         need_hp_pos=True),
    dict(dets=[[7, 7], [15, 7], [16, 7]], ref=[7, 7], n_orb=4, n_alpha=3, n_beta=3),
    dict(dets=[[7, 7], [7, 7], [0b1011, 0b10111]], ref=[7, 7], n_orb=5, n_alpha=3, n_beta=3),
]


@pytest.fixture(scope="module")
def fixture():
    return dict(np.load(os.path.join(GOLDEN, "det_batch.npz")))


def cases(fx):
    c = 0
    while f"c{c}_dets" in fx:
        n_orb, na, nb, kmax = (int(v) for v in fx[f"c{c}_shape"])
        yield c, fx[f"c{c}_dets"], fx[f"c{c}_ref"], n_orb, na, nb, kmax
        c += 1


def check_against(fx, fn):
    n = 0
    for c, d, r, n_orb, na, nb, kmax in cases(fx):
        for f, fl in enumerate(FLAGS):
            got = fn(d, r, n_orb, na, nb, kmax, *fl)
            want = {k[len(f"c{c}_f{f}_"):]: v for k, v in fx.items()
                    if k.startswith(f"c{c}_f{f}_")}
            assert set(got) == set(want), (c, f, set(got), set(want))
            for k in want:
                g = np.asarray(got[k].cpu() if hasattr(got[k], "cpu") else got[k])
                np.testing.assert_array_equal(g, want[k], err_msg=f"case {c} flags {f} {k}")
            n += 1
    assert n == 24


def errors_of(fn):
    out = []
    for e in ERROR_CASES:
        e = dict(e)
        e["dets"] = np.array(e["dets"], np.uint64)
        try:
            fn(**e)
            out.append("")
        except ValueError as err:
            out.append(str(err))
    return out


def random_dets(rng, n_orb, na, nb, B, max_exc=None, ref=None):
    """B determinants; with ref and max_exc, at most max_exc electrons of
    each spin moved from ref."""
    out = np.zeros((B, 2), np.uint64)
    for i in range(B):
        for s, ne in ((0, na), (1, nb)):
            if ref is None or max_exc is None:
                occ = rng.choice(n_orb, ne, replace=False)
            else:
                r = [o for o in range(n_orb) if (int(ref[s]) >> o) & 1]
                v = [o for o in range(n_orb) if not (int(ref[s]) >> o) & 1]
                m = int(rng.integers(0, min(max_exc, len(r), len(v)) + 1))
                gone = set(rng.choice(r, m, replace=False).tolist()) if m else set()
                occ = [o for o in r if o not in gone] + \
                    (rng.choice(v, m, replace=False).tolist() if m else [])
            for o in occ:
                out[i, s] |= np.uint64(1) << np.uint64(int(o))
    return out


# ---------------------------------------------------------------- CPU

def test_oracle_matches_golden(port, fixture):
    check_against(fixture, port.prepare_det_batch)


def test_oracle_errors_match_golden(port, fixture):
    assert errors_of(port.prepare_det_batch) == list(fixture["error_messages"])


def test_oracle_matches_reference(port, reference):
    rng = np.random.default_rng(17)
    for n_orb, na, nb, kmax in [(20, 7, 6, 5), (64, 30, 31, 70), (40, 1, 39, 3)]:
        r = random_dets(rng, n_orb, na, nb, 1)[0]
        d = random_dets(rng, n_orb, na, nb, 200)
        for fl in FLAGS:
            a = reference.prepare_det_batch(d, r, n_orb, na, nb, kmax, *fl)
            b = port.prepare_det_batch(d, r, n_orb, na, nb, kmax, *fl)
            assert set(a) == set(b)
            for k in a:
                np.testing.assert_array_equal(a[k], b[k])


def test_batch_spec_checks():
    from detnqs_b200 import det_utils as U
    with pytest.raises(ValueError, match="need_hp_pos requires hp_kmax > 0"):
        U.prepare_batch(np.zeros((1, 2), np.uint64), n_orb=4, n_alpha=0, n_beta=0,
                        ref=[0, 0], spec=U.BatchSpec(need_hp_pos=True))
    with pytest.raises(ValueError, match="bitstrings must be"):
        U.prepare_batch(np.zeros((2,), np.uint64), n_orb=4, n_alpha=0, n_beta=0,
                        ref=[0, 0], spec=U.BatchSpec())

    class M:
        batch_spec = U.BatchSpec(need_k=True)
    assert U.get_batch_spec(M()) == U.BatchSpec(need_k=True)
    assert U.get_batch_spec(object()) == U.BatchSpec()


# ---------------------------------------------------------------- GPU

@pytest.mark.gpu
def test_gpu_matches_golden(fixture):
    from detnqs_b200 import core
    check_against(fixture, core.prepare_det_batch)


@pytest.mark.gpu
def test_gpu_errors_match_golden(fixture):
    from detnqs_b200 import core
    assert errors_of(core.prepare_det_batch) == list(fixture["error_messages"])


@pytest.mark.gpu
@pytest.mark.parametrize("n_orb,na,nb,kmax,max_exc", [
    (30, 12, 12, 8, 4), (64, 32, 32, 40, None), (64, 5, 60, 3, 3), (33, 16, 17, 70, None),
    (1, 1, 0, 2, None)])
def test_gpu_matches_oracle(port, n_orb, na, nb, kmax, max_exc):
    """Larger batches: excitations beyond kmax (lists cut, mask capped),
    orbitals 32..63, kmax above a warp, a one-orbital system."""
    import torch
    from detnqs_b200 import core
    rng = np.random.default_rng(n_orb * 100 + kmax)
    r = random_dets(rng, n_orb, na, nb, 1)[0]
    d = random_dets(rng, n_orb, na, nb, 3000, max_exc=max_exc, ref=r)
    for fl in FLAGS:
        want = port.prepare_det_batch(d, r, n_orb, na, nb, kmax, *fl)
        got = core.prepare_det_batch(d, r, n_orb, na, nb, kmax, *fl)
        assert set(got) == set(want)
        for k in want:
            np.testing.assert_array_equal(got[k], want[k], err_msg=k)
        # device-resident determinants: CUDA tensors out, same values
        dd = torch.from_numpy(d.view(np.int64)).cuda()
        gd = core.prepare_det_batch(dd, r, n_orb, na, nb, kmax, *fl)
        for k in want:
            assert gd[k].is_cuda
            np.testing.assert_array_equal(gd[k].cpu().numpy(), want[k], err_msg=k)


@pytest.mark.gpu
def test_gpu_empty_and_spec():
    import torch
    from detnqs_b200 import core, det_utils as U
    out = core.prepare_det_batch(np.zeros((0, 2), np.uint64), [7, 7], 4, 3, 3, 2, True, True,
                                 True, True)
    assert out["occ"].shape == (0, 6) and out["holes_pos"].shape == (0, 2)
    d = np.array([[0b0111, 0b0111], [0b1011, 0b0111]], np.uint64)
    b = U.prepare_batch(torch.from_numpy(d.view(np.int64)).cuda(), n_orb=4, n_alpha=3,
                        n_beta=3, ref=[7, 7], spec=U.BatchSpec(hp_kmax=2, need_phase=True,
                                                               need_hp_pos=True))
    assert len(b) == 2 and b.occ.is_cuda
    assert b.aux["k"].tolist() == [0, 1]
    assert b.aux["holes"].tolist() == [[-1, -1], [2, -1]]
    assert b.aux["parts"].tolist() == [[-1, -1], [3, -1]]
    assert b.aux["hp_mask"].tolist() == [[False, False], [True, False]]
    assert b.aux["holes_pos"].tolist() == [[-1, -1], [2, -1]]
    assert b.aux["parts_pos"].tolist() == [[-1, -1], [0, -1]]
    assert b.aux["phase"].tolist() == [1, 1]
    assert len(b[1:]) == 1
