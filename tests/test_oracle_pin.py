"""Pin the oracle restatement (oracle/oracle.cpp) before trusting it.

* against the committed golden fixtures generated from the reference core;
* against the reference core itself, compiled from its sources, where the
  reference tree is present (this container);
* against the reference's own known-answer tests (tests/cpp/
  test_determinant.cpp:78-189, test_integral.cpp:65-117,
  test_hamiltonian.cpp:201-295), restated here as numbers.
"""

from __future__ import annotations

import hashlib
import os
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, assert_coo_equal, coo_of
from detnqs_b200 import synthetic as S


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _coo_sha(d):
    return _sha(d["row"].astype(np.uint32), d["col"].astype(np.uint32),
                d["val"].astype(np.float64))


@pytest.fixture(scope="module")
def small_ctx(port, golden_small):
    g = golden_small
    ctx = port.ctx_from_arrays(int(g["n_orb"]), g["h1e"], g["eri"], float(g["e_core"]))
    ctx.hb_prepare(1e-15)
    return ctx


def test_golden_small_diag(small_ctx, golden_small):
    d = small_ctx.get_ham_diag(golden_small["V"])
    np.testing.assert_array_equal(d.view(np.uint64), golden_small["diag"].view(np.uint64))


def test_golden_small_builders(small_ctx, golden_small):
    g = golden_small
    V = g["V"]
    assert_coo_equal(small_ctx.get_ham_vv(V), coo_of(g, "vv"))
    c = small_ctx.get_ham_conn(V, True, 1e-3)
    assert_coo_equal(c["H_VV"], coo_of(g, "conn_vv"))
    assert_coo_equal(c["H_VP"], coo_of(g, "conn_vp"))
    np.testing.assert_array_equal(c["det_P"], g["conn_P"])
    c = small_ctx.get_ham_conn(V, False, 1e-3)
    assert_coo_equal(c["H_VP"], coo_of(g, "connf_vp"))
    np.testing.assert_array_equal(c["det_P"], g["connf_P"])
    a = small_ctx.get_ham_conn_amp(V, g["psi"], 1e-4)
    assert_coo_equal(a["H_VV"], coo_of(g, "amp_vv"))
    assert_coo_equal(a["H_VP"], coo_of(g, "amp_vp"))
    np.testing.assert_array_equal(a["det_P"], g["amp_P"])
    b = small_ctx.get_ham_block(V[:60], g["blk_ext"])
    assert_coo_equal(b["H_VV"], coo_of(g, "blk_vv"))
    assert_coo_equal(b["H_VP"], coo_of(g, "blk_vp"))


def test_golden_small_energies_and_heff(port, small_ctx, golden_small):
    g = golden_small
    # energies are reductions whose order follows the thread schedule:
    # compared to 1e-12 Ha, not bit for bit
    e = small_ctx.compute_variational_energy(g["V"], g["psi"], True, 1e-3)
    assert abs(e - float(g["evar_hb"])) < 1e-12
    e = small_ctx.compute_variational_energy(g["V"], g["psi"], False, 1e-6)
    assert abs(e - float(g["evar_full"])) < 1e-12
    h = port.get_ham_eff(coo_of(g, "conn_vv"), coo_of(g, "conn_vp"), g["heff_hpp"],
                         float(g["heff_eref"]))
    assert_coo_equal(h, coo_of(g, "heff"))
    h = port.get_ham_eff(coo_of(g, "conn_vv"), coo_of(g, "conn_vp"), g["heff_hpp"],
                         float(g["heff_eref"]), "linear_shift", 1e-8)
    assert_coo_equal(h, coo_of(g, "heffl"))


def test_golden_small_pairs_and_table(port, small_ctx, golden_small):
    g = golden_small
    el = np.array([small_ctx.compute_elem(b, k) for b, k in zip(g["pair_bra"], g["pair_ket"])])
    np.testing.assert_array_equal(el.view(np.uint64), g["pair_elem"].view(np.uint64))
    for b, k, d, p in zip(g["pair_bra"], g["pair_ket"], g["pair_degree"], g["pair_phase"]):
        assert port.analyze(b, k) == (int(d), float(p))
    for key in g:
        if key.startswith("hb_") and key.endswith("_a"):
            i, j = (int(x) for x in key.split("_")[1:3])
            a, b, w = small_ctx.hb_row(i, j)
            ga, gb, gw = g[f"hb_{i}_{j}_a"], g[f"hb_{i}_{j}_b"], g[f"hb_{i}_{j}_w"]
            np.testing.assert_array_equal(w, gw)   # weights sorted descending
            assert set(zip(a.tolist(), b.tolist())) == set(zip(ga.tolist(), gb.tolist()))


def test_c0_checksums(port, c0_checksums):
    """Full 13-orbital workload (2241 dets) bit for bit via checksums."""
    cs = c0_checksums
    sysm = S.make_system(cs["n_orb"], cs["n_alpha"], cs["n_beta"], cs["n_chol"], cs["seed"])
    V = S.hf_sd_space(cs["n_orb"], cs["n_alpha"], cs["n_beta"])
    assert len(V) == cs["n_dets"] == 2241
    ctx = port.ctx_from_arrays(sysm.n_orb, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    assert _sha(ctx.get_ham_diag(V)) == cs["diag_sha256"]
    c = ctx.get_ham_conn(V, True, cs["eps1"])
    assert len(c["H_VV"]["val"]) == cs["conn_vv"]["nnz"] == 672561
    assert _coo_sha(c["H_VV"]) == cs["conn_vv"]["sha256"]
    assert _coo_sha(c["H_VP"]) == cs["conn_vp"]["sha256"]
    assert c["size_P"] == cs["conn_P"]["n"]
    assert _sha(c["det_P"]) == cs["conn_P"]["sha256"]


def test_fcidump_round_trip_is_exact(port):
    sysm = S.make_system(6, 2, 2, 12, 99)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "x.fcidump")
        S.write_fcidump(p, sysm)
        h1, eri, e = S.read_fcidump(p, 6)
        np.testing.assert_array_equal(h1, sysm.h1e)
        np.testing.assert_array_equal(eri, sysm.eri)
        assert e == sysm.e_core
        c1 = port.ctx_from_fcidump(p, 6)
        c2 = port.ctx_from_arrays(6, sysm.h1e, sysm.eri, sysm.e_core)
        V = S.hf_sd_space(6, 2, 2)
        np.testing.assert_array_equal(c1.get_ham_diag(V), c2.get_ham_diag(V))


# ---- known answers restated from the reference's Catch2 tests ------------

@pytest.mark.parametrize("bra,degree,phase", [
    ((0b0011, 0b0011), 0, 1.0),      # diagonal            test_determinant.cpp:83-89
    ((0b0110, 0b0011), 1, -1.0),     # single a 0->2       :91-103
    ((0b0011, 0b0110), 1, -1.0),     # single b 0->2       :105-114
    ((0b1100, 0b0011), 2, 1.0),      # double aa 01->23    :116-129
    ((0b0110, 0b1001), 2, -1.0),     # double ab           :131-139
])
def test_phase_known_answers(port, bra, degree, phase):
    ket = np.array([0b0011, 0b0011], np.uint64)
    d, p = port.analyze(np.array(bra, np.uint64), ket)
    assert d == degree and p == phase


def test_triple_has_zero_phase(port):
    d, p = port.analyze(np.array([0b1100, 0b0101], np.uint64), np.array([0b0011, 0b0011], np.uint64))
    assert d > 2 and p == 0.0   # test_determinant.cpp:141-148


def test_collector_counts(port):
    """4 orbitals, 2a2b: 8 singles + 18 doubles = 26 (test_determinant.cpp:155-189)."""
    c = port.gen_connected_dets(np.array([[0b0011, 0b0011]], np.uint64), 4)
    assert len(c) == 26


def _ref_fcidump(name, tmp_path):
    """One of the reference's FCIDUMP fixtures, rewritten from the packed
    integrals committed in tests/golden/molecules.npz (%.17e, exact), so the
    checker's FCIDUMP reader runs without the reference tree."""
    from types import SimpleNamespace
    z = np.load(os.path.join(GOLDEN, "molecules.npz"))
    n, na, nb = (int(x) for x in z[name + "_shape"])
    path = str(tmp_path / (name + ".FCIDUMP"))
    S.write_fcidump(path, SimpleNamespace(n_orb=n, n_alpha=na, n_beta=nb, n_elec=na + nb,
                                          h1e=z[name + "_h1e"], eri=z[name + "_eri"],
                                          e_core=float(z[name + "_e_nuc"])))
    return path


def test_h2_integrals_known_answers(port, tmp_path):
    """H2/6-31G values (test_integral.cpp:65-117) through the oracle."""
    ctx = port.ctx_from_fcidump(_ref_fcidump("h2_631g", tmp_path), 4)
    assert abs(ctx.get_e_nuc() - 0.26458860546) < 1e-10
    # diagonal of the HF determinant = h00 + h00 + (00|00) (alpha 0, beta 0)
    hf = np.array([[1, 1]], np.uint64)
    d = ctx.get_ham_diag(hf)[0]
    assert abs(d - (2 * -0.801833061063 + 0.422806268972)) < 1e-10


def _fci_dets(n, na, nb):
    from itertools import combinations
    A = [sum(1 << i for i in c) for c in combinations(range(n), na)]
    B = [sum(1 << i for i in c) for c in combinations(range(n), nb)]
    return np.array([[a, b] for a in A for b in B], np.uint64)


def test_h2o_fci_energy(port, tmp_path):
    """E_FCI(H2O/STO-3G) = -75.01240139 Ha, 441 dets (test_hamiltonian.cpp:282-295)."""
    ctx = port.ctx_from_fcidump(_ref_fcidump("h2o_sto3g", tmp_path), 7)
    V = _fci_dets(7, 5, 5)
    assert len(V) == 441
    h = ctx.get_ham_vv(V)
    H = np.zeros((441, 441))
    H[h["row"], h["col"]] = h["val"]
    assert np.abs(H - H.T).max() < 1e-12          # :297-316
    e = np.linalg.eigvalsh(H)[0] + ctx.get_e_nuc()
    assert abs(e - (-75.01240139)) <= 1e-7 * 75.01240139


def test_h2o_heatbath_discovery(port, tmp_path):
    """HB discovery from HF at eps1=1e-6 gives |P| in [20, 140] without HF
    (test_hamiltonian.cpp:201-225), and H_eff lowers E(HF) (:260-279)."""
    ctx = port.ctx_from_fcidump(_ref_fcidump("h2o_sto3g", tmp_path), 7)
    ctx.hb_prepare(1e-15)
    hf = np.array([[0b11111, 0b11111]], np.uint64)
    r = ctx.get_ham_conn(hf, True, 1e-6)
    assert 20 <= r["size_P"] <= 140
    assert not any((p == hf[0]).all() for p in r["det_P"])
    r = ctx.get_ham_conn(hf, True, 1e-5)
    hpp = ctx.get_ham_diag(r["det_P"])
    e_ref = ctx.get_ham_diag(hf)[0]
    h = port.get_ham_eff(r["H_VV"], r["H_VP"], hpp, e_ref, "sigma", 1e-10)
    assert h["val"][0] < r["H_VV"]["val"][0]


def test_port_matches_reference_c0(port, reference):
    """Restatement vs the compiled reference on the 13-orbital workload."""
    sysm = S.make_system(13, 5, 5, 26, 4242)
    V = S.hf_sd_space(13, 5, 5)
    psi = S.normalized_psi(len(V), 1)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "c0.fcidump")
        S.write_fcidump(p, sysm)
        a = reference.ctx_from_fcidump(p, 13)
        b = port.ctx_from_fcidump(p, 13)
        a.hb_prepare(1e-15)
        b.hb_prepare(1e-15)
        ra = a.get_ham_conn_amp(V[:600], psi[:600], 1e-6)
        rb = b.get_ham_conn_amp(V[:600], psi[:600], 1e-6)
        assert_coo_equal(ra["H_VV"], rb["H_VV"])
        assert_coo_equal(ra["H_VP"], rb["H_VP"])
        np.testing.assert_array_equal(ra["det_P"], rb["det_P"])
        la = a.get_local_connections(V[:40], True, 1e-6)
        lb = b.get_local_connections(V[:40], True, 1e-6)
        np.testing.assert_array_equal(la["offsets"], lb["offsets"])
        pa = a.compute_pt2(V[:300], psi[:300] / np.linalg.norm(psi[:300]), -100.0, True, 1e-5)
        pb = b.compute_pt2(V[:300], psi[:300] / np.linalg.norm(psi[:300]), -100.0, True, 1e-5)
        assert pa["n_ext"] == pb["n_ext"]
        assert abs(pa["e_pt2_external"] - pb["e_pt2_external"]) < 1e-12
        ga = a.gen_perturbative_dets(V[:50], psi[:50], "static", 1e-5)
        gb = b.gen_perturbative_dets(V[:50], psi[:50], "static", 1e-5)
        np.testing.assert_array_equal(ga, gb)
