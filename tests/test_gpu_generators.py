"""GPU parity of the determinant-space generators, local connectivity and
EN-PT2 against the oracle restatement (itself pinned to the reference)."""

from __future__ import annotations

import numpy as np
import pytest

from detnqs_b200 import synthetic as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(port):
    from detnqs_b200 import core
    sysm = S.make_system(13, 5, 5, 26, 777)
    V = S.hf_sd_space(13, 5, 5)
    ctx = core.IntCtx.from_arrays(13, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    octx = port.ctx_from_arrays(13, sysm.h1e, sysm.eri, sysm.e_core)
    octx.hb_prepare(1e-15)
    psi = S.normalized_psi(len(V), 12)
    return core, ctx, octx, V, psi


def test_gen_connected(setup, port):
    core, ctx, octx, V, psi = setup
    np.testing.assert_array_equal(core.gen_connected_dets(V[:1], 13),
                                  port.gen_connected_dets(V[:1], 13))
    np.testing.assert_array_equal(core.gen_connected_dets(V[:40], 13),
                                  port.gen_connected_dets(V[:40], 13))
    four = np.array([[0b0011, 0b0011]], np.uint64)
    assert len(core.gen_connected_dets(four, 4)) == 26     # test_determinant.cpp:155-189


@pytest.mark.parametrize("mode,eps", [("none", 0.0), ("static", 1e-5), ("static", 1e-3),
                                      ("dynamic", 1e-5)])
def test_gen_perturbative(setup, mode, eps):
    core, ctx, octx, V, psi = setup
    sub, p = V[:80], psi[:80]
    got = core.gen_perturbative_dets(sub, 13, ctx, p, mode=mode, eps1=eps)
    want = octx.gen_perturbative_dets(sub, p, mode, eps)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("use_hb,eps", [(True, 1e-6), (True, 1e-3), (False, 1e-6)])
def test_local_connections(setup, use_hb, eps):
    core, ctx, octx, V, psi = setup
    sub = V[100:160]
    got = core.get_local_connections(sub, ctx, 13, use_hb, eps)
    want = octx.get_local_connections(sub, use_hb, eps)
    # every row in the reference's order: singles, then doubles in table
    # order (ties as std::sort leaves them) or in for_each_double's order
    np.testing.assert_array_equal(got["offsets"], want["offsets"])
    np.testing.assert_array_equal(got["dets"], want["dets"])
    np.testing.assert_array_equal(got["values"].view(np.uint64), want["values"].view(np.uint64))


@pytest.mark.parametrize("use_hb", [True, False])
def test_pt2(setup, use_hb):
    core, ctx, octx, V, psi = setup
    sub = V[:400]
    c = psi[:400] / np.linalg.norm(psi[:400])
    e_ref = -60.0
    got = core.compute_pt2(sub, c, ctx, 13, e_ref, use_hb, 1e-5)
    want = octx.compute_pt2(sub, c, e_ref, use_hb, 1e-5)
    assert got["n_ext"] == want["n_ext"]
    assert abs(got["e_pt2_external"] - want["e_pt2_external"]) < 1e-12
    assert abs(got["e_pt2_internal"] - want["e_pt2_internal"]) <= 1e-12 * max(1.0, abs(want["e_pt2_internal"]))


def test_operator_layer(setup):
    """detnqs.operator mirror: builders + operators against SciPy."""
    core, ctx, octx, V, psi = setup
    from types import SimpleNamespace
    from detnqs_b200 import operator as op
    system = SimpleNamespace(int_ctx=ctx, n_orb=13)
    space = SimpleNamespace(V_dets=V[:500])
    vv = op.build_vv_hamiltonian(system, space)
    ref = octx.get_ham_vv(V[:500])
    A = np.zeros((500, 500))
    A[ref["row"], ref["col"]] = ref["val"]
    x = psi[:500]
    y = op.build_vv_operator(vv, jax_dtype=np.float64)(x).V
    np.testing.assert_allclose(y, A @ x, rtol=0, atol=1e-11)
    np.testing.assert_array_equal(vv.diagonals.V, np.diag(A))
    prox, P = op.build_proxy_hamiltonian(system, space, screening="static", screen_eps=1e-5)
    want = octx.get_ham_conn(V[:500], True, 1e-5)
    np.testing.assert_array_equal(P, want["det_P"])
    xp = S.normalized_psi(len(P), 3)
    out = op.build_proxy_operator(prox, jax_dtype=np.float64)(x, xp)
    import scipy.sparse as sp
    VP = sp.csr_matrix((want["H_VP"]["val"], (want["H_VP"]["row"], want["H_VP"]["col"])),
                       shape=want["H_VP"]["shape"])
    VV = sp.csr_matrix((want["H_VV"]["val"], (want["H_VV"]["row"], want["H_VV"]["col"])),
                       shape=want["H_VV"]["shape"])
    dp = octx.get_ham_diag(P)
    np.testing.assert_allclose(out.V, VV @ x + VP @ xp, rtol=0, atol=1e-10)
    np.testing.assert_allclose(out.P, VP.T @ x + dp * xp, rtol=0, atol=1e-10)
    eff = op.build_effective_hamiltonian(system, prox, -60.0)
    h = octx.chk.get_ham_eff(want["H_VV"], want["H_VP"], dp, -60.0)
    B = eff.ham_vv.tocoo()
    np.testing.assert_array_equal(B.row, h["row"])
    np.testing.assert_array_equal(B.col, h["col"])
    np.testing.assert_array_equal(B.data.view(np.uint64), h["val"].view(np.uint64))
    prox2, P2 = op.build_proxy_hamiltonian(system, SimpleNamespace(V_dets=V[:30]),
                                           screening="none")
    np.testing.assert_array_equal(P2, octx.gen_perturbative_dets(V[:30]))
