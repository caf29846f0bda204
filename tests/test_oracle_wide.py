"""Pin the two-word restatement (oracle/wide.cpp) to the reference core.

The reference holds a spin string in one uint64, so it cannot check
100-orbital determinants directly.  Here, for n <= 64, the W = 1 and W = 2
(high words zero) instances of the restatement must reproduce the
reference's get_ham_conn (static heat-bath) and get_ham_conn_amp (dynamic
amplitude screening) bit for bit: H_VV, H_VP and the sorted P set.  CPU only.
"""

from __future__ import annotations

import os
import tempfile

import numpy as np
import pytest

from conftest import assert_coo_equal

from detnqs_b200 import synthetic as S


def widen(d: np.ndarray) -> np.ndarray:
    out = np.zeros((len(d), 4), np.uint64)
    out[:, 0] = d[:, 0]
    out[:, 2] = d[:, 1]
    return out


def narrow(d: np.ndarray) -> np.ndarray:
    assert not d[:, 1].any() and not d[:, 3].any()
    return np.ascontiguousarray(d[:, [0, 2]])


def cases():
    c0 = S.make_system(13, 5, 5, 26, 20251)
    yield "c0", c0, S.hf_sd_space(13, 5, 5)
    # 64 orbitals: bit 63 is reachable and the last table rows are used
    big = S.make_system(64, 3, 3, 8, 611)
    yield "n64", big, S.heat_bath_sample(big, 60, 612, max_level=4)


@pytest.fixture(scope="module", params=["c0", "n64"])
def system(request, reference):
    from oracle import WideChecker
    for name, sysm, V in cases():
        if name == request.param:
            break
    with tempfile.TemporaryDirectory() as d:
        fd = os.path.join(d, "sys.fcidump")
        S.write_fcidump(fd, sysm)
        ref = reference.ctx_from_fcidump(fd, sysm.n_orb)
    ref.hb_prepare(1e-15)
    wide = WideChecker(sysm.n_orb, sysm.h1e, sysm.eri, sysm.e_core)
    wide.hb_prepare(1e-15)
    return sysm, V, ref, wide


@pytest.mark.parametrize("words", [1, 2])
@pytest.mark.parametrize("eps1", [1e-6, 1e-2])
def test_static_heatbath_matches_reference(system, words, eps1):
    sysm, V, ref, wide = system
    r = ref.get_ham_conn(V, use_heatbath=True, eps1=eps1)
    w = wide.build(V if words == 1 else widen(V), eps1=eps1)
    assert_coo_equal(w["H_VV"], r["H_VV"])
    assert_coo_equal(w["H_VP"], r["H_VP"])
    P = w["det_P"] if words == 1 else narrow(w["det_P"])
    np.testing.assert_array_equal(P, r["det_P"])


@pytest.mark.parametrize("words", [1, 2])
@pytest.mark.parametrize("eps1", [1e-5, 1e-3])
def test_dynamic_amplitude_matches_reference(system, words, eps1):
    sysm, V, ref, wide = system
    psi = S.normalized_psi(len(V), 77)
    r = ref.get_ham_conn_amp(V, psi, eps1=eps1)
    w = wide.build(V if words == 1 else widen(V), psi, eps1=eps1)
    assert_coo_equal(w["H_VV"], r["H_VV"])
    assert_coo_equal(w["H_VP"], r["H_VP"])
    P = w["det_P"] if words == 1 else narrow(w["det_P"])
    np.testing.assert_array_equal(P, r["det_P"])


def test_row_subset_is_a_slice_of_the_full_build(system):
    """Building rows [r0, r1) gives those rows' entries (P columns mapped
    back to determinants)."""
    sysm, V, ref, wide = system
    W2 = widen(V)
    full = wide.build(W2, eps1=1e-3)
    part = wide.build(W2, eps1=1e-3, rows=(5, 40))

    def rows_of(res, lo, hi):
        vp = res["H_VP"]
        sel = (vp["row"] >= lo) & (vp["row"] < hi)
        keys = [tuple(x) for x in res["det_P"][vp["col"][sel]].tolist()]
        return sorted(zip(vp["row"][sel].tolist(), keys, vp["val"][sel].view(np.uint64).tolist()))

    assert rows_of(full, 5, 40) == rows_of(part, 5, 40)


def test_diag_and_elements_match_reference(system):
    sysm, V, ref, wide = system
    d = ref.get_ham_diag(V)
    np.testing.assert_array_equal(wide.diag(widen(V)).view(np.uint64), d.view(np.uint64))
    rng = np.random.default_rng(3)
    for _ in range(40):
        i, j = rng.integers(0, len(V), 2)
        e = ref.compute_elem(V[i], V[j])
        assert wide.elem(widen(V[i:i + 1]), widen(V[j:j + 1])) == e


def test_wide_sampler_and_packing():
    """Two-word packing round trip and a 100-orbital sample that reaches
    both words."""
    sysm = S.make_system(100, 6, 6, 12, 5)
    V = S.heat_bath_sample_wide(sysm, 500, 6, max_level=3)
    a, b = S.unpack_wide(V, 100)
    assert (a.sum(1) == 6).all() and (b.sum(1) == 6).all()
    occa = np.nonzero(a)[1].reshape(-1, 6)
    occb = np.nonzero(b)[1].reshape(-1, 6)
    np.testing.assert_array_equal(S.pack_wide(occa, occb), V)
    assert len(np.unique(V, axis=0)) == len(V)
    assert (V[:, 1] != 0).any() and (V[:, 3] != 0).any()
