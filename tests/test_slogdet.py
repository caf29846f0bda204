"""Batched log-determinant (the reference's fused log-det kernels,
csrc/ffi/logdet_cuda.cu, through detnqs/models/slogdet.py).

The reference checks its kernel against XLA's slogdet (tests/python/
test_logdet.py:27-66: |d sign|, |d log|det||, |d grad| below 1e-8 in FP64
and 1e-4 in FP32, on N(0,1) + n I matrices).  Here the checker is LAPACK's
slogdet and inverse through numpy in FP64, with the same FP64 bounds; FP32
results are held to 1e-4 relative to the FP64 values.  Matrices without the
diagonal shift and with sign flips exercise the pivoting and the sign.
"""

from __future__ import annotations

import numpy as np
import pytest


def batch(rng, B, n, shift=True, dtype=np.float64):
    a = rng.normal(size=(B, n, n))
    if shift:
        a += np.eye(n) * n
    a[::3, 0, :] *= -1.0   # negative determinants too
    return a.astype(dtype)


def reference(a):
    a64 = a.astype(np.float64)
    s, l = np.linalg.slogdet(a64)
    return s, l, np.swapaxes(np.linalg.inv(a64), -1, -2)


# ---------------------------------------------------------------- CPU

def test_argument_checks():
    from detnqs_b200 import slogdet as L
    with pytest.raises(TypeError, match="Unsupported dtype"):
        L.slogdet(np.zeros((2, 4, 4), np.int32))
    with pytest.raises(ValueError, match="Expected square matrix"):
        L.slogdet(np.zeros((2, 4, 5)))
    with pytest.raises(ValueError, match=r"outside \[2, 64\] range"):
        L.slogdet(np.zeros((2, 65, 65)))
    with pytest.raises(ValueError, match="Batch shape mismatch"):
        L.slogdet_grad(np.zeros((2, 4, 4)), np.zeros(3))


# ---------------------------------------------------------------- GPU

@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 3, 8, 16, 17, 24, 31, 32, 33, 48, 63, 64])
@pytest.mark.parametrize("shift", [True, False])
def test_slogdet_fp64(n, shift):
    from detnqs_b200 import slogdet as L
    rng = np.random.default_rng(n * 7 + shift)
    a = batch(rng, 37, n, shift)
    s, l = L.slogdet(a)
    s0, l0, g0 = reference(a)
    np.testing.assert_array_equal(s, s0)
    assert np.max(np.abs(l - l0)) < 1e-8
    cot = rng.normal(size=37)
    g = L.slogdet_grad(a, cot)
    assert np.max(np.abs(g - cot[:, None, None] * g0)) < 1e-8 * max(1.0, np.abs(g0).max())


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 10, 24, 33, 64])
def test_slogdet_fp32(n):
    from detnqs_b200 import slogdet as L
    rng = np.random.default_rng(n)
    a = batch(rng, 41, n, True, np.float32)
    s, l = L.slogdet(a)
    assert s.dtype == np.float32 and l.dtype == np.float32
    s0, l0, g0 = reference(a)
    np.testing.assert_array_equal(s, s0)
    assert np.max(np.abs(l - l0) / np.maximum(1.0, np.abs(l0))) < 1e-4
    g = L.slogdet_grad(a, np.ones(41, np.float32))
    assert np.max(np.abs(g - g0)) < 1e-4 * np.abs(g0).max()


@pytest.mark.gpu
def test_singular_and_batch_shapes():
    """A zero column gives sign 0, log|det| -inf and a zero gradient, beside
    regular matrices of the same batch; a multi-dimensional batch keeps its
    shape."""
    from detnqs_b200 import slogdet as L
    rng = np.random.default_rng(5)
    a = batch(rng, 24, 12).reshape(4, 6, 12, 12)
    a[1, 2, :, 5] = 0.0
    s, l = L.slogdet(a)
    assert s.shape == (4, 6) and s[1, 2] == 0.0 and l[1, 2] == -np.inf
    g = L.slogdet_grad(a, np.ones((4, 6)))
    assert np.all(g[1, 2] == 0.0)
    mask = np.ones((4, 6), bool)
    mask[1, 2] = False
    s0, l0, g0 = reference(a[mask])
    np.testing.assert_array_equal(s[mask], s0)
    assert np.max(np.abs(l[mask] - l0)) < 1e-8
    assert np.max(np.abs(g[mask] - g0)) < 1e-8
    from detnqs_b200 import native as N
    with pytest.raises(ValueError, match="Batch size out of int32 range"):
        N.check(N.lib.dnq_slogdet(a.ctypes.data, 0, 12, N.F64, s.ctypes.data, l.ctypes.data,
                                  0, None))


@pytest.mark.gpu
def test_autograd_and_resident():
    """CUDA tensors in and out, and torch autograd through the kernels: the
    gradient of sum(log|det|) is A^{-T}."""
    import torch
    from detnqs_b200 import slogdet as L
    rng = np.random.default_rng(9)
    a = batch(rng, 300, 20)
    t = torch.from_numpy(a).cuda().requires_grad_(True)
    s, l = L.slogdet_autograd(t)
    assert s.is_cuda and l.is_cuda
    l.sum().backward()
    s0, l0, g0 = reference(a)
    np.testing.assert_array_equal(s.detach().cpu().numpy(), s0)
    assert np.max(np.abs(l.detach().cpu().numpy() - l0)) < 1e-8
    assert np.max(np.abs(t.grad.cpu().numpy() - g0)) < 1e-8
