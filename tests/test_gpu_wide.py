"""Two-word determinants (up to 128 orbitals) on the GPU.

* At 13 orbitals the two-word build equals the one-word build bit for bit
  (H_VV, H_VP, P), under static and dynamic screening.
* At 100 orbitals it equals the two-word restatement in oracle/wide.cpp
  (which is itself pinned to the reference core at n <= 64) bit for bit.
* Diagonal elements of P, downfolding on the device handle, and the
  one-word entry points' refusal of a 100-orbital context.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_coo_equal

from detnqs_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def widen(d: np.ndarray) -> np.ndarray:
    out = np.zeros((len(d), 4), np.uint64)
    out[:, 0] = d[:, 0]
    out[:, 2] = d[:, 1]
    return out


def hf_dominated_psi(n: int, seed: int, tail: float) -> np.ndarray:
    """HF amplitude 1 and a Gaussian tail of scale ``tail`` (row 0 is HF)."""
    rng = np.random.default_rng(seed)
    psi = tail * rng.normal(size=n)
    psi[0] = 1.0
    return psi / np.linalg.norm(psi)


@pytest.mark.parametrize("eps1", [1e-6, 1e-3])
@pytest.mark.parametrize("dynamic", [False, True])
def test_wide_equals_narrow_at_13_orbitals(eps1, dynamic):
    from detnqs_b200 import core
    from detnqs_b200 import wide as Wd
    sysm = S.make_system(13, 5, 5, 26, 20251)
    V = S.hf_sd_space(13, 5, 5)
    ctx = core.IntCtx.from_arrays(13, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    wctx = Wd.IntCtxWide.from_arrays(13, sysm.h1e, sysm.eri, sysm.e_core)
    wctx.hb_prepare(1e-15)
    if dynamic:
        psi = S.normalized_psi(len(V), 8)
        a = core.get_ham_conn_amp(V, psi, ctx, 13, eps1=eps1)
        b = Wd.get_ham_conn_amp_wide(widen(V), psi, wctx, 13, eps1=eps1)
    else:
        a = core.get_ham_conn(V, ctx, 13, use_heatbath=True, eps1=eps1)
        b = Wd.get_ham_conn_wide(widen(V), wctx, 13, eps1=eps1)
    assert_coo_equal(b["H_VV"], a["H_VV"])
    assert_coo_equal(b["H_VP"], a["H_VP"])
    np.testing.assert_array_equal(b["det_P"], widen(a["det_P"]))
    np.testing.assert_array_equal(Wd.get_ham_diag_wide(widen(V), wctx).view(np.uint64),
                                  core.get_ham_diag(V, ctx).view(np.uint64))


@pytest.fixture(scope="module")
def n100():
    """100 orbitals, 10 alpha / 10 beta, K = 200; 150 heat-bath-sampled
    determinants (about half reach orbitals >= 64)."""
    from oracle import WideChecker
    from detnqs_b200 import wide as Wd
    sysm = S.make_system(100, 10, 10, 200, 4100)
    V = S.heat_bath_sample_wide(sysm, 150, 4101, max_level=3)
    ctx = Wd.IntCtxWide.from_arrays(100, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    chk = WideChecker(100, sysm.h1e, sysm.eri, sysm.e_core)
    chk.hb_prepare(1e-15)
    return sysm, V, ctx, chk


def test_wide_equals_oracle_at_100_orbitals(n100):
    from detnqs_b200 import wide as Wd
    sysm, V, ctx, chk = n100
    assert (V[:, 1] != 0).any() and (V[:, 3] != 0).any()
    psi = hf_dominated_psi(len(V), 5, 2e-5)
    g = Wd.get_ham_conn_amp_wide(V, psi, ctx, 100, eps1=1e-5)
    o = chk.build(V, psi, eps1=1e-5)
    assert g["size_P"] == o["size_P"] > 0
    np.testing.assert_array_equal(g["det_P"], o["det_P"])
    assert_coo_equal(g["H_VV"], o["H_VV"])
    assert_coo_equal(g["H_VP"], o["H_VP"])
    # static screening with a cut that keeps part of every table row
    g = Wd.get_ham_conn_wide(V[1:40], ctx, 100, eps1=0.45)
    o = chk.build(V[1:40], eps1=0.45)
    np.testing.assert_array_equal(g["det_P"], o["det_P"])
    assert_coo_equal(g["H_VV"], o["H_VV"])
    assert_coo_equal(g["H_VP"], o["H_VP"])
    np.testing.assert_array_equal(Wd.get_ham_diag_wide(V, ctx).view(np.uint64),
                                  chk.diag(V).view(np.uint64))


def test_downfolding_on_wide_handle(n100):
    """H_eff from the device handle equals the reference downfolding
    (restated) applied to the oracle's blocks, bit for bit in FP64; the FP32
    form (FP32 H_VP values, float-float accumulation, FP64 shift) moves the
    lowest eigenvalue by at most 1e-6 Ha.

    e_ref is the variational energy of V and D^-1 is sigma-regularised with
    epsilon = 0.1 Ha (ham_eff.cpp:35-56): the synthetic spectrum has P
    determinants within micro-Hartrees of e_ref, whose 1/d terms would
    otherwise dominate H_eff."""
    from oracle import Checker
    from detnqs_b200 import native as N
    from detnqs_b200 import wide as Wd
    sysm, V, ctx, chk = n100
    psi = hf_dominated_psi(len(V), 6, 2e-5)
    H = Wd.build_wide(ctx, V, psi, n_orb=100, eps1=1e-5)
    hpp = Wd.p_diag(H, ctx)
    P = H.dets_p()
    np.testing.assert_array_equal(hpp.view(np.uint64), chk.diag(P).view(np.uint64))

    def sym(M):
        A = M.toarray()
        return 0.5 * (A + A.T)

    e_ref = float(np.linalg.eigvalsh(sym(H.to_scipy(0)))[0])
    E64 = Wd.ham_eff_wide(H, hpp, e_ref, epsilon=0.1, precision=N.F64)
    E32 = Wd.ham_eff_wide(H, hpp, e_ref, epsilon=0.1, precision=N.F32)
    o = chk.build(V, psi, eps1=1e-5)
    ref = Checker.port().get_ham_eff(o["H_VV"], o["H_VP"], chk.diag(o["det_P"]), e_ref,
                                     "sigma", 0.1)
    assert_coo_equal(E64.to_coo(0), ref)
    low64 = np.linalg.eigvalsh(sym(E64.to_scipy(0)))[0]
    low32 = np.linalg.eigvalsh(sym(E32.to_scipy(0)))[0]
    # The synthetic integrals give the HF row about 1.2e6 doubles whose
    # second-order sum is ~ -2400 Ha; that row (over 65536 entries) keeps its
    # FP64 values in FP32 mode, so the bound is the absolute 1e-6 Ha.
    assert abs(low32 - low64) <= 1e-6, (low32, low64)
    for h in (H, E64, E32):
        h.close()


def test_one_word_entry_points_refuse_wide_context(n100):
    from detnqs_b200 import core
    sysm, V, ctx, chk = n100
    with pytest.raises(ValueError, match="more than 64 orbitals"):
        core.get_ham_diag(np.zeros((1, 2), np.uint64), ctx)


def test_symmetric_part_and_lanczos(n100):
    """0.5 (H + H^T) on the device equals the same sum on the host bit for
    bit, and device Lanczos finds its lowest eigenvalue."""
    from detnqs_b200 import eigen as E
    from detnqs_b200 import native as N
    from detnqs_b200 import wide as Wd
    sysm, V, ctx, chk = n100
    psi = hf_dominated_psi(len(V), 7, 2e-5)
    H = Wd.build_wide(ctx, V, psi, n_orb=100, eps1=1e-5)
    hpp = Wd.p_diag(H, ctx)
    num, den = H.local_energy(psi)
    Heff = Wd.ham_eff_wide(H, hpp, num / den, epsilon=0.1, precision=N.F64)
    Hs = E.symmetric_part(Heff)
    A = Heff.to_scipy(0).toarray()
    ref = 0.5 * (A + A.T)
    np.testing.assert_array_equal(Hs.to_scipy(0).toarray(), ref)
    lam, steps = E.lowest_eigenvalue(Hs)
    exact = np.linalg.eigvalsh(ref)[0]
    assert abs(lam - exact) <= 1e-10 * abs(exact), (lam, exact, steps)
    for h in (H, Heff, Hs):
        h.close()
