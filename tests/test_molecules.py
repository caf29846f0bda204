"""Real molecules from the reference's own FCIDUMP fixtures.

The integrals of H2O/STO-3G, H2O/6-31G, Cr2 (24e, 30o) and N2/cc-pVDZ are
committed in tests/golden/molecules.npz, and the reference core's outputs on
them as checksums in tests/golden/molecule_checksums.json
(tests/golden/make_molecules.py made both from the reference tree).  Unlike
the synthetic integrals these have point-group zeros and many exactly tied
heat-bath weights, so they check the order the reference leaves ties in
(std::ranges::sort, hb_table.cpp:133) and everything that inherits it:
get_local_connections (local_conn.cpp:36-142) row by row in order.

CPU tests pin the oracle restatement to the checksums; GPU tests hold the
CUDA path to the same checksums and to the reference's known answer
E_FCI(H2O/STO-3G) = -75.01240139 Ha (test_hamiltonian.cpp:282-295).
"""

from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

E_FCI_H2O = -75.01240139


def _sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def coo_sha(d: dict) -> dict:
    return {"nnz": int(len(d["val"])), "shape": [int(x) for x in d["shape"]],
            "sha256": _sha(np.asarray(d["row"], np.uint32), np.asarray(d["col"], np.uint32),
                           np.asarray(d["val"], np.float64))}


def conn_sha(c: dict) -> dict:
    return {"n": int(len(c["values"])),
            "sha256": _sha(np.asarray(c["offsets"], np.int32), np.asarray(c["dets"], np.uint64),
                           np.asarray(c["values"], np.float64))}


def hb_rows_sha(row_of, nso: int) -> dict:
    h = hashlib.sha256()
    ties = total = 0
    for i in range(1, nso):
        for j in range(i):
            a, b, w = row_of(i, j)
            h.update(np.asarray(a, np.int32).tobytes())
            h.update(np.asarray(b, np.int32).tobytes())
            h.update(np.asarray(w, np.float64).tobytes())
            total += len(w)
            ties += bool(len(w) > 1 and np.any(w[1:] == w[:-1]))
    return {"entries": total, "rows_with_ties": ties, "sha256": h.hexdigest()}


@pytest.fixture(scope="module")
def mols():
    z = np.load(os.path.join(GOLDEN, "molecules.npz"))
    out = {}
    for key in z.files:
        if key.endswith("_shape"):
            name = key[:-6]
            n, na, nb = (int(x) for x in z[key])
            out[name] = {"n_orb": n, "n_alpha": na, "n_beta": nb, "h1e": z[name + "_h1e"],
                         "eri": z[name + "_eri"], "e_nuc": float(z[name + "_e_nuc"])}
    return out


@pytest.fixture(scope="module")
def sums():
    with open(os.path.join(GOLDEN, "molecule_checksums.json")) as f:
        return json.load(f)


def hf_sd(m):
    from detnqs_b200 import synthetic as S
    return S.hf_sd_space(m["n_orb"], m["n_alpha"], m["n_beta"])


def fci_dets(n, na, nb):
    from itertools import combinations
    A = [sum(1 << i for i in c) for c in combinations(range(n), na)]
    B = [sum(1 << i for i in c) for c in combinations(range(n), nb)]
    return np.array([[a, b] for a in A for b in B], np.uint64)


def cr2_space(m, sums):
    from types import SimpleNamespace
    from detnqs_b200 import synthetic as S
    sysm = SimpleNamespace(n_orb=m["n_orb"], n_alpha=m["n_alpha"], n_beta=m["n_beta"],
                           h1e=m["h1e"], eri=m["eri"])
    V = S.heat_bath_sample(sysm, sums["cr2_dets"], 17)
    assert _sha(V.astype(np.uint64)) == sums["molecules"]["cr2_24e30o"]["vv_rows"]["space_sha256"]
    return V


def psi_for(n):
    from detnqs_b200 import synthetic as S
    return S.normalized_psi(n, 31)


# ---------------------------------------------------------------------------
# CPU: the oracle restatement against the reference's checksums
# ---------------------------------------------------------------------------

@pytest.fixture(scope="module")
def port_ctx(port, mols):
    ctxs = {}
    for name, m in mols.items():
        c = port.ctx_from_arrays(m["n_orb"], m["h1e"], m["eri"], m["e_nuc"])
        c.hb_prepare(1e-15)
        ctxs[name] = c
    return ctxs


def test_port_fci_energy_h2o(port, mols):
    m = mols["h2o_sto3g"]
    c = port.ctx_from_arrays(7, m["h1e"], m["eri"], m["e_nuc"])
    V = fci_dets(7, 5, 5)
    h = c.get_ham_vv(V)
    H = np.zeros((441, 441))
    H[h["row"], h["col"]] = h["val"]
    e = np.linalg.eigvalsh(H)[0] + c.get_e_nuc()
    assert abs(e - E_FCI_H2O) <= 1e-7 * abs(E_FCI_H2O)


@pytest.mark.parametrize("name", ["h2o_sto3g", "h2o_631g", "cr2_24e30o", "n2_ccpvdz"])
def test_port_heatbath_rows_in_reference_order(port_ctx, mols, sums, name):
    want = sums["molecules"][name]["hb_rows"]
    assert want["rows_with_ties"] > 0          # these molecules do have ties
    got = hb_rows_sha(port_ctx[name].hb_row, 2 * mols[name]["n_orb"])
    assert got == want


@pytest.mark.parametrize("name", ["h2o_sto3g", "h2o_631g", "cr2_24e30o", "n2_ccpvdz"])
@pytest.mark.parametrize("use_hb", [True, False])
def test_port_local_connections_in_order(port_ctx, mols, sums, name, use_hb):
    rec = sums["molecules"][name]
    sub = hf_sd(mols[name])[rec["local_conn_rows"]]
    got = port_ctx[name].get_local_connections(sub, use_hb, sums["local_eps"])
    assert conn_sha(got) == rec["local_conn_hb" if use_hb else "local_conn_full"]


@pytest.mark.parametrize("name", ["h2o_sto3g", "h2o_631g"])
def test_port_builders_on_molecules(port, port_ctx, mols, sums, name):
    rec = sums["molecules"][name]
    c = port_ctx[name]
    V = hf_sd(mols[name])
    psi = psi_for(len(V))
    conn = c.get_ham_conn(V, True, sums["conn_eps"])
    assert coo_sha(conn["H_VV"]) == rec["conn"]["H_VV"]
    assert coo_sha(conn["H_VP"]) == rec["conn"]["H_VP"]
    assert _sha(conn["det_P"].astype(np.uint64)) == rec["conn"]["det_P_sha256"]
    amp = c.get_ham_conn_amp(V, psi, sums["amp_eps"])
    assert coo_sha(amp["H_VV"]) == rec["conn_amp"]["H_VV"]
    assert coo_sha(amp["H_VP"]) == rec["conn_amp"]["H_VP"]
    hpp = c.get_ham_diag(amp["det_P"])
    eff = port.get_ham_eff(amp["H_VV"], amp["H_VP"], hpp, rec["eff"]["e_ref"])
    assert coo_sha(eff) == {k: rec["eff"][k] for k in ("nnz", "shape", "sha256")}
    e = c.compute_variational_energy(V, psi, True, sums["amp_eps"])
    assert abs(e - rec["e_var_hb"]) <= 1e-12 * abs(e)


def test_port_cr2_rows(port_ctx, mols, sums):
    rec = sums["molecules"]["cr2_24e30o"]["vv_rows"]
    V = cr2_space(mols["cr2_24e30o"], sums)
    rows = [r["row"] for r in rec["rows"]]
    blk = port_ctx["cr2_24e30o"].vv_hb_rows(V, rows, sums["cr2_eps"])
    for r in rec["rows"]:
        sel = blk["row"] == r["row"]
        cols, vals = blk["col"][sel], blk["val"][sel]
        o = np.argsort(cols, kind="stable")
        assert int(sel.sum()) == r["nnz"]
        assert _sha(cols[o].astype(np.uint32), vals[o].astype(np.float64)) == r["sha256"]


# ---------------------------------------------------------------------------
# GPU: the CUDA path against the same checksums
# ---------------------------------------------------------------------------

@pytest.fixture(scope="module")
def gpu_ctx(mols):
    from detnqs_b200 import core
    ctxs = {}
    for name, m in mols.items():
        c = core.IntCtx.from_arrays(m["n_orb"], m["h1e"], m["eri"], m["e_nuc"])
        c.hb_prepare(1e-15)
        ctxs[name] = c
    yield ctxs
    for c in ctxs.values():
        c.close()


@pytest.mark.gpu
def test_gpu_fci_energy_h2o(mols, tmp_path):
    """E_FCI(H2O/STO-3G) from get_ham_block over the 441-determinant FCI
    space, read through the FCIDUMP reader (test_hamiltonian.cpp:282-295)."""
    from types import SimpleNamespace
    from detnqs_b200 import core
    from detnqs_b200 import synthetic as S
    m = mols["h2o_sto3g"]
    path = str(tmp_path / "h2o.FCIDUMP")
    S.write_fcidump(path, SimpleNamespace(n_orb=7, n_alpha=5, n_beta=5, n_elec=10,
                                          h1e=m["h1e"], eri=m["eri"], e_core=m["e_nuc"]))
    ctx = core.IntCtx(path, 7)
    assert ctx.get_e_nuc() == m["e_nuc"]
    V = fci_dets(7, 5, 5)
    blk = core.get_ham_block(V, None, ctx, 7)
    h = blk["H_VV"]
    H = np.zeros((441, 441))
    H[h["row"], h["col"]] = h["val"]
    assert np.abs(H - H.T).max() < 1e-12                       # :297-316
    e = np.linalg.eigvalsh(H)[0] + ctx.get_e_nuc()
    assert abs(e - E_FCI_H2O) <= 1e-7 * abs(E_FCI_H2O)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["h2o_sto3g", "h2o_631g", "cr2_24e30o", "n2_ccpvdz"])
def test_gpu_heatbath_rows_in_reference_order(gpu_ctx, mols, sums, name):
    got = hb_rows_sha(gpu_ctx[name].hb_row, 2 * mols[name]["n_orb"])
    assert got == sums["molecules"][name]["hb_rows"]


@pytest.mark.gpu
def test_gpu_tie_order_follows_hb_threshold(gpu_ctx, port, mols):
    """hb_prepare with a threshold above the table's own: the reference's
    table then holds only the heavier entries, and its sort orders their
    ties among those alone."""
    from detnqs_b200 import core
    m = mols["n2_ccpvdz"]
    c = core.IntCtx.from_arrays(m["n_orb"], m["h1e"], m["eri"], m["e_nuc"])
    o = port.ctx_from_arrays(m["n_orb"], m["h1e"], m["eri"], m["e_nuc"])
    for thr in (1e-6, 1e-15):
        c.hb_prepare(thr)
        o.hb_prepare(thr)
        assert hb_rows_sha(c.hb_row, 2 * m["n_orb"]) == hb_rows_sha(o.hb_row, 2 * m["n_orb"])
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["h2o_sto3g", "h2o_631g", "cr2_24e30o", "n2_ccpvdz"])
@pytest.mark.parametrize("use_hb", [True, False])
def test_gpu_local_connections_in_order(gpu_ctx, mols, sums, name, use_hb):
    from detnqs_b200 import core
    rec = sums["molecules"][name]
    m = mols[name]
    sub = hf_sd(m)[rec["local_conn_rows"]]
    got = core.get_local_connections(sub, gpu_ctx[name], m["n_orb"], use_hb, sums["local_eps"])
    assert conn_sha(got) == rec["local_conn_hb" if use_hb else "local_conn_full"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["h2o_sto3g", "h2o_631g"])
def test_gpu_builders_on_molecules(gpu_ctx, mols, sums, name):
    from detnqs_b200 import core
    rec = sums["molecules"][name]
    m = mols[name]
    ctx, n = gpu_ctx[name], m["n_orb"]
    V = hf_sd(m)
    psi = psi_for(len(V))
    conn = core.get_ham_conn(V, ctx, n, use_heatbath=True, eps1=sums["conn_eps"])
    assert coo_sha(conn["H_VV"]) == rec["conn"]["H_VV"]
    assert coo_sha(conn["H_VP"]) == rec["conn"]["H_VP"]
    assert conn["size_P"] == rec["conn"]["size_P"]
    assert _sha(conn["det_P"].astype(np.uint64)) == rec["conn"]["det_P_sha256"]
    amp = core.get_ham_conn_amp(V, psi, ctx, n, eps1=sums["amp_eps"])
    assert coo_sha(amp["H_VV"]) == rec["conn_amp"]["H_VV"]
    assert coo_sha(amp["H_VP"]) == rec["conn_amp"]["H_VP"]
    assert _sha(amp["det_P"].astype(np.uint64)) == rec["conn_amp"]["det_P_sha256"]
    hpp = core.get_ham_diag(amp["det_P"], ctx)
    eff = core.get_ham_eff(amp["H_VV"], amp["H_VP"], hpp, rec["eff"]["e_ref"])
    assert coo_sha(eff) == {k: rec["eff"][k] for k in ("nnz", "shape", "sha256")}
    for use_hb, key in ((True, "e_var_hb"), (False, "e_var_full")):
        e = core.compute_variational_energy(V, psi, ctx, n, use_hb, sums["amp_eps"])
        assert abs(e - rec[key]) <= 1e-12 * abs(rec[key])


@pytest.mark.gpu
def test_gpu_cr2_rows(gpu_ctx, mols, sums):
    """A heat-bath-sampled Cr2 space (20000 determinants): the screened V->V
    block built on the GPU (string-group path), row by row against the
    reference's rows."""
    from detnqs_b200 import device, native
    rec = sums["molecules"]["cr2_24e30o"]["vv_rows"]
    m = mols["cr2_24e30o"]
    V = cr2_space(m, sums)
    H = device.build(gpu_ctx["cr2_24e30o"], V, n_orb=30, policy=native.POLICY_STATIC,
                     use_heatbath=True, eps1=sums["cr2_eps"], want_vp=False)
    rp, cols, vals = H.to_csr_arrays(0)
    for r in rec["rows"]:
        a, b = int(rp[r["row"]]), int(rp[r["row"] + 1])
        c, v = cols[a:b], vals[a:b]
        o = np.argsort(c, kind="stable")
        assert b - a == r["nnz"]
        assert _sha(c[o].astype(np.uint32), v[o].astype(np.float64)) == r["sha256"]
    H.close()
