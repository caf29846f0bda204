"""The build's own radix sort (determinant sets, P discovery, row
canonicalisation) against a stable host sort: same order for 64-bit keys
and (alpha, beta) pairs, with many equal keys, sizes around the 2048-key
tiles, and only the significant bits visited."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _order(keys: np.ndarray, bits) -> np.ndarray:
    from detnqs_b200 import native as N
    words = 1 if keys.ndim == 1 else keys.shape[1]
    k = np.ascontiguousarray(keys, np.uint64)
    b = (C.c_int * words)(*bits)
    out = np.empty(len(k), np.uint32)
    N.check(N.lib.dnq_sort_order(k.ctypes.data, len(k), words, b, out.ctypes.data, 0, None))
    return out


@pytest.mark.parametrize("n", [1, 2, 31, 2047, 2048, 2049, 100003, 1 << 20])
def test_u64_keys_stable(n):
    rng = np.random.default_rng(n)
    for bits in (5, 26, 60):
        keys = rng.integers(0, 1 << bits, size=n, dtype=np.uint64)
        np.testing.assert_array_equal(_order(keys, [bits]), np.argsort(keys, kind="stable"))


@pytest.mark.parametrize("n_orb", [6, 13, 30, 64])
def test_determinant_pairs_stable(n_orb):
    rng = np.random.default_rng(n_orb)
    n = 300_001
    hi = (1 << n_orb) - 1 if n_orb < 64 else (1 << 64) - 1
    a = rng.integers(0, min(hi, 1 << 20), size=n, dtype=np.uint64) & np.uint64(hi)
    b = rng.integers(0, min(hi, 1 << 12), size=n, dtype=np.uint64) & np.uint64(hi)
    if n_orb == 64:
        a = a | (np.uint64(1) << np.uint64(63)) * (rng.integers(0, 2, n).astype(np.uint64))
    keys = np.stack([a, b], 1)
    want = np.lexsort((b, a))          # stable: alpha, then beta, then position
    np.testing.assert_array_equal(_order(keys, [n_orb, n_orb]), want)
