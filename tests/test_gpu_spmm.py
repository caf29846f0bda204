"""H applied to several amplitude vectors in one pass (dnq_ham_spmv_multi,
dnq_ham_local_energy_multi) against the single-vector operator: every
column bit for bit (same lanes per row, same accumulation order), energies
and local energies bit for bit, FP64 against SciPy's CSR matvec (the
reference's H.psi, detnqs/operator/kernel.py:75-78) within 1e-12."""

from __future__ import annotations

import numpy as np
import pytest

from detnqs_b200 import synthetic as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ham():
    from detnqs_b200 import core, device, native
    sysm = S.make_system(16, 5, 5, 32, 99)
    V = S.heat_bath_sample(sysm, 20000, 3)
    ctx = core.IntCtx.from_arrays(16, sysm.h1e, sysm.eri, sysm.e_core)
    ctx.hb_prepare(1e-15)
    H = device.build(ctx, V, n_orb=16, policy=native.POLICY_STATIC, use_heatbath=True,
                     eps1=1e-6, want_vp=False)
    yield native, H
    H.close()
    ctx.close()


def _X(n, k, seed):
    X = np.random.default_rng(seed).normal(size=(n, k))
    return X / np.linalg.norm(X, axis=0)


@pytest.mark.parametrize("prec_name", ["f64", "f32"])
@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 8, 11])
def test_columns_equal_single_vector(ham, prec_name, k):
    import torch
    native, H = ham
    prec = native.F64 if prec_name == "f64" else native.F32
    X = torch.from_numpy(_X(H.n_v, k, k)).cuda()
    Y = H.spmv_multi(X, precision=prec)
    torch.cuda.synchronize()
    Yh = Y.cpu().numpy()
    for j in range(k):
        y = H.spmv(X[:, j].contiguous(), precision=prec).cpu().numpy()
        np.testing.assert_array_equal(Yh[:, j].view(np.uint64), y.view(np.uint64))
    if prec == native.F64:
        A = H.to_scipy(0)
        ref = A @ X.cpu().numpy()
        np.testing.assert_allclose(Yh, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("prec_name", ["f64", "f32"])
@pytest.mark.parametrize("k", [3, 8, 9])
def test_energies_equal_single_vector(ham, prec_name, k):
    import torch
    native, H = ham
    prec = native.F64 if prec_name == "f64" else native.F32
    X = torch.from_numpy(_X(H.n_v, k, 40 + k)).cuda()
    eloc = torch.empty_like(X)
    out = H.local_energy_multi(X, eloc=eloc, precision=prec)
    torch.cuda.synchronize()
    for j in range(k):
        el = torch.empty(H.n_v, dtype=torch.float64, device=X.device)
        num, den = H.local_energy(X[:, j].contiguous(), eloc=el, precision=prec)
        assert np.float64(out[j, 0]).view(np.uint64) == np.float64(num).view(np.uint64)
        assert np.float64(out[j, 1]).view(np.uint64) == np.float64(den).view(np.uint64)
        np.testing.assert_array_equal(eloc[:, j].cpu().numpy().view(np.uint64),
                                      el.cpu().numpy().view(np.uint64))


def test_host_buffers(ham):
    native, H = ham
    X = _X(H.n_v, 4, 7)
    Y = H.spmv_multi(X, precision=native.F32)
    for j in range(4):
        np.testing.assert_array_equal(Y[:, j], H.spmv(X[:, j].copy(), precision=native.F32))
    out = H.local_energy_multi(X)
    num, den = H.local_energy(X[:, 2].copy())
    assert out[2, 0] == num and out[2, 1] == den
