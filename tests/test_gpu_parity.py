"""GPU parity: libdetnqs_b200 (through its C ABI) against the oracle and the
golden fixtures made from the reference core.

Bar: integer results (connectivity, columns, P order, phases, degrees) are
bit-exact; FP64 matrix elements are bit-exact too (the kernels keep the
reference's summation order); energies agree to 1e-12 Ha; the FP32
operator agrees with FP64 to |dE| <= 1e-6 Ha.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import assert_coo_equal, coo_of
from detnqs_b200 import synthetic as S

pytestmark = pytest.mark.gpu

ENERGY_TOL = 1e-12     # Ha, FP64 energies
FP32_DE_TOL = 1e-6     # Ha, FP32-compensated operator vs FP64


@pytest.fixture(scope="module")
def core():
    from detnqs_b200 import core as C
    return C


@pytest.fixture(scope="module")
def gctx(core, golden_small):
    g = golden_small
    ctx = core.IntCtx.from_arrays(int(g["n_orb"]), g["h1e"], g["eri"], float(g["e_core"]))
    ctx.hb_prepare(1e-15)
    return ctx


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _coo_sha(d):
    return _sha(d["row"].astype(np.uint32), d["col"].astype(np.uint32),
                d["val"].astype(np.float64))


# ---------------------------------------------------------------------------
# Slater-Condon primitives
# ---------------------------------------------------------------------------

def test_pairs_degree_phase_and_elements(core, gctx, golden_small):
    g = golden_small
    deg, ph = core.excitations(g["pair_bra"], g["pair_ket"])
    np.testing.assert_array_equal(deg, g["pair_degree"])
    np.testing.assert_array_equal(ph, g["pair_phase"])
    el = core.get_ham_elems(g["pair_bra"], g["pair_ket"], gctx)
    np.testing.assert_array_equal(el.view(np.uint64), g["pair_elem"].view(np.uint64))


def test_known_answer_phases(core):
    ket = np.array([[0b0011, 0b0011]] * 6, np.uint64)
    bra = np.array([[0b0011, 0b0011], [0b0110, 0b0011], [0b0011, 0b0110],
                    [0b1100, 0b0011], [0b0110, 0b1001], [0b1100, 0b0101]], np.uint64)
    deg, ph = core.excitations(bra, ket)
    np.testing.assert_array_equal(deg[:5], [0, 1, 1, 2, 2])
    np.testing.assert_array_equal(ph, [1.0, -1.0, -1.0, 1.0, -1.0, 0.0])
    assert deg[5] > 2


def test_diag_bits(core, gctx, golden_small):
    d = core.get_ham_diag(golden_small["V"], gctx)
    np.testing.assert_array_equal(d.view(np.uint64), golden_small["diag"].view(np.uint64))


def test_heatbath_rows(gctx, golden_small):
    g = golden_small
    for key in g:
        if key.startswith("hb_") and key.endswith("_a"):
            i, j = (int(x) for x in key.split("_")[1:3])
            a, b, w = gctx.hb_row(i, j)
            np.testing.assert_array_equal(w, g[f"hb_{i}_{j}_w"])
            assert set(zip(a.tolist(), b.tolist())) == set(
                zip(g[f"hb_{i}_{j}_a"].tolist(), g[f"hb_{i}_{j}_b"].tolist()))


# ---------------------------------------------------------------------------
# Builders vs golden (bit-exact)
# ---------------------------------------------------------------------------

def test_get_ham_vv(core, gctx, golden_small):
    g = golden_small
    assert_coo_equal(core.get_ham_vv(g["V"], gctx, int(g["n_orb"])), coo_of(g, "vv"))


def test_get_ham_conn_static(core, gctx, golden_small):
    g = golden_small
    r = core.get_ham_conn(g["V"], gctx, int(g["n_orb"]), use_heatbath=True, eps1=1e-3)
    assert_coo_equal(r["H_VV"], coo_of(g, "conn_vv"))
    assert_coo_equal(r["H_VP"], coo_of(g, "conn_vp"))
    np.testing.assert_array_equal(r["det_P"], g["conn_P"])
    assert r["size_P"] == len(g["conn_P"])


def test_get_ham_conn_unscreened(core, gctx, golden_small):
    g = golden_small
    r = core.get_ham_conn(g["V"], gctx, int(g["n_orb"]), use_heatbath=False, eps1=1e-3)
    assert_coo_equal(r["H_VV"], coo_of(g, "connf_vv"))
    assert_coo_equal(r["H_VP"], coo_of(g, "connf_vp"))
    np.testing.assert_array_equal(r["det_P"], g["connf_P"])


def test_get_ham_conn_amp(core, gctx, golden_small):
    g = golden_small
    r = core.get_ham_conn_amp(g["V"], g["psi"], gctx, int(g["n_orb"]), eps1=1e-4)
    assert_coo_equal(r["H_VV"], coo_of(g, "amp_vv"))
    assert_coo_equal(r["H_VP"], coo_of(g, "amp_vp"))
    np.testing.assert_array_equal(r["det_P"], g["amp_P"])


def test_get_ham_block(core, gctx, golden_small):
    g = golden_small
    r = core.get_ham_block(g["V"][:60], g["blk_ext"], int_ctx=gctx, n_orb=int(g["n_orb"]))
    assert_coo_equal(r["H_VV"], coo_of(g, "blk_vv"))
    assert_coo_equal(r["H_VP"], coo_of(g, "blk_vp"))
    np.testing.assert_array_equal(r["det_P"], g["blk_ext"])
    r = core.get_ham_block(g["V"][:60], None, int_ctx=gctx, n_orb=int(g["n_orb"]))
    assert "det_P" not in r and len(r["H_VP"]["val"]) == 0


def test_variational_energy(core, gctx, golden_small):
    g = golden_small
    n = int(g["n_orb"])
    e = core.compute_variational_energy(g["V"], g["psi"], gctx, n, True, 1e-3)
    assert abs(e - float(g["evar_hb"])) < ENERGY_TOL
    e = core.compute_variational_energy(g["V"], g["psi"], gctx, n, False, 1e-6)
    assert abs(e - float(g["evar_full"])) < ENERGY_TOL


def test_get_ham_eff_fp64_bits(core, golden_small):
    g = golden_small
    h = core.get_ham_eff(coo_of(g, "conn_vv"), coo_of(g, "conn_vp"), g["heff_hpp"],
                         float(g["heff_eref"]))
    assert_coo_equal(h, coo_of(g, "heff"))
    h = core.get_ham_eff(coo_of(g, "conn_vv"), coo_of(g, "conn_vp"), g["heff_hpp"],
                         float(g["heff_eref"]), "linear_shift", 1e-8)
    assert_coo_equal(h, coo_of(g, "heffl"))


def test_get_ham_eff_fp32_lowest_eigenvalue(core, golden_small):
    g = golden_small
    ref = coo_of(g, "heff")
    h = core.get_ham_eff(coo_of(g, "conn_vv"), coo_of(g, "conn_vp"), g["heff_hpp"],
                         float(g["heff_eref"]), precision="fp32")
    n = ref["shape"][0]
    A = np.zeros((n, n))
    A[ref["row"], ref["col"]] = ref["val"]
    B = np.zeros((n, n))
    B[h["row"], h["col"]] = h["val"]
    dE = abs(np.linalg.eigvalsh(A)[0] - np.linalg.eigvalsh(B)[0])
    assert dE <= FP32_DE_TOL


# ---------------------------------------------------------------------------
# Full 13-orbital workload (2241 dets): checksums of the reference outputs
# ---------------------------------------------------------------------------

@pytest.fixture(scope="module")
def c0(core, c0_checksums):
    cs = c0_checksums
    sysm = S.make_system(cs["n_orb"], cs["n_alpha"], cs["n_beta"], cs["n_chol"], cs["seed"])
    V = S.hf_sd_space(cs["n_orb"], cs["n_alpha"], cs["n_beta"])
    ctx = core.IntCtx.from_arrays(sysm.n_orb, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    return cs, sysm, V, ctx


def test_c0_conn_bits(core, c0):
    cs, sysm, V, ctx = c0
    assert _sha(core.get_ham_diag(V, ctx)) == cs["diag_sha256"]
    r = core.get_ham_conn(V, ctx, 13, use_heatbath=True, eps1=cs["eps1"])
    assert len(r["H_VV"]["val"]) == cs["conn_vv"]["nnz"]
    assert len(r["H_VP"]["val"]) == cs["conn_vp"]["nnz"]
    assert _coo_sha(r["H_VV"]) == cs["conn_vv"]["sha256"]
    assert _coo_sha(r["H_VP"]) == cs["conn_vp"]["sha256"]
    assert r["size_P"] == cs["conn_P"]["n"]
    assert _sha(r["det_P"]) == cs["conn_P"]["sha256"]


def test_c0_amp_bits_and_energy(core, c0):
    cs, sysm, V, ctx = c0
    psi = S.normalized_psi(len(V), cs["psi_seed"])
    r = core.get_ham_conn_amp(V, psi, ctx, 13, eps1=1e-6)
    assert _coo_sha(r["H_VV"]) == cs["amp_vv"]["sha256"]
    assert _coo_sha(r["H_VP"]) == cs["amp_vp"]["sha256"]
    assert _sha(r["det_P"]) == cs["amp_P"]["sha256"]
    e = core.compute_variational_energy(V, psi, ctx, 13, True, 1e-6)
    assert abs(e - cs["evar_hb_1e-6"]) < ENERGY_TOL


def test_c0_heff_bits(core, c0):
    cs, sysm, V, ctx = c0
    r = core.get_ham_conn(V, ctx, 13, use_heatbath=True, eps1=cs["eps1"])
    hpp = core.get_ham_diag(r["det_P"], ctx)
    h = core.get_ham_eff(r["H_VV"], r["H_VP"], hpp, cs["heff_e_ref"])
    assert len(h["val"]) == cs["heff"]["nnz"]
    assert _coo_sha(h) == cs["heff"]["sha256"]


# ---------------------------------------------------------------------------
# H.psi, local energy, proxy operator
# ---------------------------------------------------------------------------

def test_spmv_local_energy_and_fp32(core, c0):
    import scipy.sparse as sp
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    cs, sysm, V, ctx = c0
    H = D.build(ctx, V, n_orb=13, policy=N.POLICY_STATIC, use_heatbath=True, eps1=1e-8)
    ref = H.to_scipy(0)
    psi = S.normalized_psi(len(V), 9)
    y = H.spmv(psi)
    y_ref = ref.dot(psi)
    np.testing.assert_allclose(y, y_ref, rtol=0, atol=1e-12 * np.abs(y_ref).max())
    num, den = H.local_energy(psi)
    e64 = num / den
    assert abs(e64 - psi @ y_ref / (psi @ psi)) < ENERGY_TOL
    eloc = np.empty(len(V))
    H.local_energy(psi, eloc=eloc)
    np.testing.assert_allclose(eloc, y_ref / psi, rtol=1e-11)
    n32, d32 = H.local_energy(psi, precision=N.F32)
    assert abs(n32 / d32 - e64) <= FP32_DE_TOL
    y32 = H.spmv(psi, precision=N.F32)
    assert np.abs(y32 - y_ref).max() < 1e-5
    # proxy operator against SciPy (kernel.py:127-139)
    R = core.get_ham_conn(V, ctx, 13, use_heatbath=True, eps1=1e-8)
    vp = sp.csr_matrix((R["H_VP"]["val"], (R["H_VP"]["row"], R["H_VP"]["col"])),
                       shape=R["H_VP"]["shape"])
    xp = S.normalized_psi(R["size_P"], 4)
    dp = core.get_ham_diag(R["det_P"], ctx)
    yv, yp = H.proxy_spmv(psi, xp, dp)
    yv_ref = ref.dot(psi) + vp.dot(xp)
    yp_ref = vp.T.dot(psi) + dp * xp
    np.testing.assert_allclose(yv, yv_ref, rtol=0, atol=1e-11 * np.abs(yv_ref).max())
    np.testing.assert_allclose(yp, yp_ref, rtol=0, atol=1e-11 * np.abs(yp_ref).max())
    yv32, yp32 = H.proxy_spmv(psi, xp, dp, precision=N.F32)
    assert np.abs(yv32 - yv_ref).max() < 1e-5 and np.abs(yp32 - yp_ref).max() < 1e-4
    H.close()


def test_spmv_device_tensors(core, c0):
    import torch
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    cs, sysm, V, ctx = c0
    H = D.build(ctx, torch.from_numpy(V.view(np.int64)).cuda(), n_orb=13,
                policy=N.POLICY_KNOWN_SETS, want_vp=False)
    psi = torch.from_numpy(S.normalized_psi(len(V), 2)).cuda()
    y = H.spmv(psi)
    assert y.is_cuda
    ref = H.to_scipy(0).dot(psi.cpu().numpy())
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    H.close()


# ---------------------------------------------------------------------------
# The bench's single-system workload itself: 30 orbitals, 12 alpha / 12 beta,
# K = 60, 10^6 heat-bath-sampled determinants, eps1 = 1e-6, default arena
# chunk.  Rows longer than a chunk go through the long-row kernels.
# ---------------------------------------------------------------------------

def test_bench_workload_rows_match_oracle(core, port):
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    sysm = S.make_system(30, 12, 12, 60, 1001)
    V = S.heat_bath_sample(sysm, 1_000_000, 2002)
    ctx = core.IntCtx.from_arrays(30, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    H = D.build(ctx, V, n_orb=30, policy=N.POLICY_STATIC, use_heatbath=True, eps1=1e-6,
                want_vp=False)
    rp, cols, vals = H.to_csr_arrays(0)
    lens = np.diff(rp)
    assert lens.max() > 16384                   # rows over one arena chunk exist
    rows = np.unique(np.concatenate([np.argsort(-lens, kind="stable")[:16],
                                     np.random.default_rng(1).choice(len(V), 64,
                                                                     replace=False)]))
    octx = port.ctx_from_arrays(30, sysm.h1e, sysm.eri, sysm.e_core)
    octx.hb_prepare(1e-15)
    o = octx.vv_hb_rows(V, rows, 1e-6)
    got = {"row": np.repeat(rows, lens[rows]).astype(np.uint32),
           "col": np.concatenate([cols[rp[r]:rp[r + 1]] for r in rows]),
           "val": np.concatenate([vals[rp[r]:rp[r + 1]] for r in rows]),
           "shape": (len(V), len(V))}
    # copy_csr returns each row sorted by column, as the COO the oracle gives
    assert_coo_equal(got, o)
    H.close()
    ctx.close()


# ---------------------------------------------------------------------------
# Larger heat-bath-sampled space (30 orbitals): row subset vs the oracle
# ---------------------------------------------------------------------------

def test_large_space_rows_match_oracle(core, port):
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    sysm = S.make_system(30, 12, 12, 60, 31)
    V = S.heat_bath_sample(sysm, 20000, 5)
    ctx = core.IntCtx.from_arrays(30, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    H = D.build(ctx, V, n_orb=30, policy=N.POLICY_STATIC, use_heatbath=True, eps1=1e-6,
                want_vp=False)
    rp, cols, vals = H.to_csr_arrays(0)
    octx = port.ctx_from_arrays(30, sysm.h1e, sysm.eri, sysm.e_core)
    octx.hb_prepare(1e-15)
    rows = np.random.default_rng(0).choice(len(V), 64, replace=False)
    rows.sort()
    o = octx.vv_hb_rows(V, rows, 1e-6)
    got = {"row": np.repeat(rows, rp[rows + 1] - rp[rows]).astype(np.uint32),
           "col": np.concatenate([cols[rp[r]:rp[r + 1]] for r in rows]),
           "val": np.concatenate([vals[rp[r]:rp[r + 1]] for r in rows]),
           "shape": (len(V), len(V))}
    assert_coo_equal(got, o)
    # exact Hermiticity of the whole block (both triangles computed independently)
    A = H.to_scipy(0)
    assert (A - A.T).count_nonzero() == 0
    H.close()


# ---------------------------------------------------------------------------
# Edge cases the reference reports
# ---------------------------------------------------------------------------

def test_edge_cases(core, gctx, golden_small):
    g = golden_small
    n = int(g["n_orb"])
    V = g["V"]
    empty = np.zeros((0, 2), np.uint64)
    r = core.get_ham_vv(empty, gctx, n)
    assert len(r["val"]) == 0
    r = core.get_ham_conn(empty, gctx, n, True, 1e-3)
    assert r["size_P"] == 0
    assert len(core.get_ham_diag(empty, gctx)) == 0
    with pytest.raises(ValueError, match="duplicate"):
        core.get_ham_vv(np.concatenate([V[:5], V[:1]]), gctx, n)
    with pytest.raises(ValueError, match="size mismatch"):
        core.get_ham_conn_amp(V, g["psi"][:-1], gctx, n)
    ctx2 = core.IntCtx.from_arrays(n, g["h1e"], g["eri"], float(g["e_core"]))
    with pytest.raises(ValueError, match="Heat-Bath table not initialized"):
        core.get_ham_conn(V, ctx2, n, use_heatbath=True)
    with pytest.raises(ValueError, match="Heat-Bath table not initialized"):
        core.get_ham_conn_amp(V, g["psi"], ctx2, n)
    bad = V[:3].copy()
    bad[0, 0] |= np.uint64(1 << 20)
    with pytest.raises(ValueError):
        core.get_ham_diag(bad, gctx)
    with pytest.raises(ValueError, match="invalid reg_type"):
        core.get_ham_eff(coo_of(g, "conn_vv"), coo_of(g, "conn_vp"), g["heff_hpp"], 0.0,
                         reg_type="bogus")
    one = V[:1]
    r = core.get_ham_conn(one, gctx, n, True, 1e-3)
    assert r["H_VV"]["shape"] == (1, 1) and r["size_P"] > 0
    # empty P space: H_eff is H_VV canonicalised (ham_eff.cpp:72-77)
    h = core.get_ham_eff(coo_of(g, "vv"), {"row": [], "col": [], "val": [], "shape": (0, 0)},
                         np.zeros(0), -1.0)
    assert_coo_equal(h, coo_of(g, "vv"))


@pytest.mark.parametrize("policy,use_hb,eps", [(0, False, 0.0), (1, True, 1e-6), (1, True, 1e-3),
                                               (1, False, 1e-6), (2, True, 1e-6)])
@pytest.mark.parametrize("n_orb", [20, 40])
def test_string_groups_match_candidate_walk(core, policy, use_hb, eps, n_orb):
    """V->V-only builds take the string-group matcher (32-bit scans at 20
    orbitals, 64-bit at 40); the candidate walk (forced by
    DNQ_OPT_FORCE_WALK) must give the identical block."""
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    if n_orb == 20:
        sysm = S.make_system(20, 7, 6, 40, 17)
        V = S.heat_bath_sample(sysm, 30000, 9)
    else:
        sysm = S.make_system(40, 8, 8, 80, 19)
        V = S.heat_bath_sample(sysm, 15000, 11)
    psi = S.normalized_psi(len(V), 4)
    ctx = core.IntCtx.from_arrays(n_orb, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    kw = dict(n_orb=n_orb, policy=policy, use_heatbath=use_hb, eps1=eps, want_vp=False,
              psi=psi if policy == 2 else None)
    A = D.build(ctx, V, **kw)
    N.check(N.lib.dnq_set_option(1, 1))
    try:
        B = D.build(ctx, V, **kw)
    finally:
        N.check(N.lib.dnq_set_option(1, 0))
    assert_coo_equal(A.to_coo(0), B.to_coo(0))
    A.close()
    B.close()


@pytest.mark.parametrize("policy", [1, 2])
def test_partc_walks_identical(core, policy):
    """Short alpha-single groups of the opposite-spin doubles walked packed
    (default) and one group at a time (DNQ_OPT_PARTC_GROUPWALK) give the same
    block with the same entries in the same row order: the FP64 H.psi over
    the unsorted rows agrees bit for bit."""
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    sysm = S.make_system(24, 9, 8, 48, 29)
    V = S.heat_bath_sample(sysm, 40000, 12)
    psi = S.normalized_psi(len(V), 6)
    ctx = core.IntCtx.from_arrays(24, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    kw = dict(n_orb=24, policy=policy, use_heatbath=True, eps1=1e-6, want_vp=False,
              psi=psi if policy == 2 else None)
    # long alpha groups (> 128 members and > the 8 x 16 beta singles of a
    # row) take the presence rows, the rest the short-group walks
    counts = np.unique(V[:, 0], return_counts=True)[1]
    assert (counts > 128).sum() >= 10 and (counts <= 128).sum() >= 1000
    A = D.build(ctx, V, **kw)
    ya = A.spmv(psi)
    N.check(N.lib.dnq_set_option(N.OPT_PARTC_GROUPWALK, 1))
    try:
        B = D.build(ctx, V, **kw)
    finally:
        N.check(N.lib.dnq_set_option(N.OPT_PARTC_GROUPWALK, 0))
    yb = B.spmv(psi)
    assert A.candidates == B.candidates
    np.testing.assert_array_equal(ya.view(np.uint64), yb.view(np.uint64))
    assert_coo_equal(A.to_coo(0), B.to_coo(0))
    A.close()
    B.close()


@pytest.mark.parametrize("chunk,cap", [(0, 0), (64, 0), (0, 5000)])
def test_build_f32_copy_matches(core, chunk, cap):
    """DNQ_OPT_BUILD_F32 writes the FP32 copy and the diagonal while the rows
    are compacted (short rows, and long rows with small chunks); the two-pass
    fallback (tiny arena) leaves them to the first FP32 use.  FP32 H.psi is
    bit-identical to the copy made on first use, before and after a sort of
    the rows."""
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    sysm = S.make_system(18, 6, 6, 36, 23)
    V = S.heat_bath_sample(sysm, 12000, 3)
    psi = S.normalized_psi(len(V), 4)
    ctx = core.IntCtx.from_arrays(18, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    kw = dict(n_orb=18, policy=1, use_heatbath=True, eps1=1e-6, want_vp=False)
    N.check(N.lib.dnq_set_option(N.OPT_ARENA_CHUNK, chunk))
    N.check(N.lib.dnq_set_option(N.OPT_ARENA_CAP, cap))
    try:
        A = D.build(ctx, V, **kw)
        N.check(N.lib.dnq_set_option(N.OPT_BUILD_F32, 1))
        B = D.build(ctx, V, **kw)
    finally:
        N.check(N.lib.dnq_set_option(N.OPT_BUILD_F32, 0))
        N.check(N.lib.dnq_set_option(N.OPT_ARENA_CHUNK, 0))
        N.check(N.lib.dnq_set_option(N.OPT_ARENA_CAP, 0))
    ya = A.spmv(psi, precision=N.F32)
    yb = B.spmv(psi, precision=N.F32)
    np.testing.assert_array_equal(ya.view(np.uint64), yb.view(np.uint64))
    np.testing.assert_array_equal(A.spmv(psi).view(np.uint64), B.spmv(psi).view(np.uint64))
    assert_coo_equal(A.to_coo(0), B.to_coo(0))   # sorts the rows
    np.testing.assert_array_equal(A.spmv(psi, precision=N.F32).view(np.uint64),
                                  B.spmv(psi, precision=N.F32).view(np.uint64))
    A.close()
    B.close()


@pytest.mark.parametrize("chunk,cap", [(64, 0), (512, 0), (0, 5000)])
def test_arena_paths_match(core, chunk, cap):
    """Small warp chunks force row restarts and the long-row pass; a tiny
    arena forces the exact two-pass fallback.  All give the same block."""
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    sysm = S.make_system(18, 6, 6, 36, 23)
    V = S.heat_bath_sample(sysm, 12000, 3)
    ctx = core.IntCtx.from_arrays(18, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    kw = dict(n_orb=18, policy=1, use_heatbath=True, eps1=1e-7, want_vp=False)
    A = D.build(ctx, V, **kw)
    N.check(N.lib.dnq_set_option(2, chunk))
    N.check(N.lib.dnq_set_option(3, cap))
    try:
        ctx2 = core.IntCtx.from_arrays(18, sysm.h1e, sysm.eri, sysm.e_core)
        ctx2.hb_prepare(1e-15)
        B = D.build(ctx2, V, **kw)
    finally:
        N.check(N.lib.dnq_set_option(2, 0))
        N.check(N.lib.dnq_set_option(3, 0))
    assert_coo_equal(A.to_coo(0), B.to_coo(0))
    # H.psi agrees with the sorted copy
    x = S.normalized_psi(len(V), 1)
    ref = A.to_scipy(0).dot(x)
    np.testing.assert_allclose(B.spmv(x), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    A.close()
    B.close()


def test_spmv_every_lane_and_slot_count(core):
    """H.psi for every (lanes per row, slots per lane): for fixed lanes the
    result does not depend on the slots in flight (same order of
    accumulation), and every form agrees with SciPy."""
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    sysm = S.make_system(18, 6, 6, 36, 23)
    V = S.heat_bath_sample(sysm, 12000, 3)
    ctx = core.IntCtx.from_arrays(18, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    H = D.build(ctx, V, n_orb=18, policy=1, use_heatbath=True, eps1=1e-7, want_vp=False)
    x = S.normalized_psi(len(V), 5)
    ref = H.to_scipy(0).dot(x)
    scale = np.abs(ref).max()
    for G in (4, 8, 16, 32):
        H.set_option(N.OPT_SPMV_LANES, G)
        first = {}
        for U in (1, 2, 4):
            H.set_option(N.OPT_SPMV_UNROLL, U)
            for prec in (N.F64, N.F32):
                y = H.spmv(x, precision=prec)
                if prec in first:
                    np.testing.assert_array_equal(y, first[prec])
                else:
                    first[prec] = y
                tol = 1e-12 if prec == N.F64 else 1e-6
                np.testing.assert_allclose(y, ref, rtol=0, atol=tol * scale)
    H.close()


def test_options_are_copied_per_handle(core):
    """dnq_set_option changes the defaults of handles built afterwards only;
    dnq_ham_set_option changes one handle's H.psi shape and no other's."""
    from detnqs_b200 import device as D
    from detnqs_b200 import native as N
    sysm = S.make_system(18, 6, 6, 36, 23)
    V = S.heat_bath_sample(sysm, 12000, 3)
    ctx = core.IntCtx.from_arrays(18, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    kw = dict(n_orb=18, policy=1, use_heatbath=True, eps1=1e-7, want_vp=False)
    x = S.normalized_psi(len(V), 5)
    A = D.build(ctx, V, **kw)
    B = D.build(ctx, V, **kw)
    y_auto = A.spmv(x)
    B.set_option(N.OPT_SPMV_LANES, 4)
    B.set_option(N.OPT_SPMV_UNROLL, 1)
    y4 = B.spmv(x)
    np.testing.assert_array_equal(A.spmv(x), y_auto)       # A untouched
    # a default set afterwards reaches neither existing handle
    N.check(N.lib.dnq_set_option(N.OPT_SPMV_LANES, 32))
    try:
        np.testing.assert_array_equal(A.spmv(x), y_auto)
        np.testing.assert_array_equal(B.spmv(x), y4)
        C = D.build(ctx, V, **kw)                           # takes the new default
        C.set_option(N.OPT_SPMV_UNROLL, 1)
        y32 = C.spmv(x)
        A.set_option(N.OPT_SPMV_LANES, 32)
        A.set_option(N.OPT_SPMV_UNROLL, 1)
        np.testing.assert_array_equal(A.spmv(x), y32)
    finally:
        N.check(N.lib.dnq_set_option(N.OPT_SPMV_LANES, 0))
    with pytest.raises(ValueError, match="lanes per row"):
        A.set_option(N.OPT_SPMV_LANES, 3)
    with pytest.raises(ValueError, match="only the H.psi options"):
        A.set_option(N.OPT_ARENA_CHUNK, 64)
    for h in (A, B, C):
        h.close()
