"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on
CPU only (no CUDA calls)."""

from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# The reference source tree, when $DETNQS_REFERENCE_ROOT names one (tests
# that read its files skip without it).
REFERENCE_TREE = os.environ.get("DETNQS_REFERENCE_ROOT", "")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_port():
    from oracle import PORT_LIB
    if not os.path.exists(PORT_LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"],
                       check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def port():
    """The oracle restatement (built on demand from oracle/oracle.cpp)."""
    _ensure_port()
    from oracle import Checker
    return Checker.port()


@pytest.fixture(scope="session")
def reference():
    from oracle import Checker
    if not Checker.reference_available():
        pytest.skip("reference core not compiled here (oracle/_ref)")
    return Checker.reference()


@pytest.fixture(scope="session")
def golden_small():
    return dict(np.load(os.path.join(GOLDEN, "golden_small.npz")))


@pytest.fixture(scope="session")
def c0_checksums():
    with open(os.path.join(GOLDEN, "c0_checksums.json")) as f:
        return json.load(f)


def coo_of(g: dict, prefix: str) -> dict:
    return {"row": g[prefix + "_row"], "col": g[prefix + "_col"], "val": g[prefix + "_val"],
            "shape": tuple(int(x) for x in g[prefix + "_shape"])}


def assert_coo_equal(a: dict, b: dict, bits: bool = True, atol: float = 0.0):
    assert tuple(a["shape"]) == tuple(b["shape"]), (a["shape"], b["shape"])
    assert len(a["val"]) == len(b["val"]), (len(a["val"]), len(b["val"]))
    np.testing.assert_array_equal(np.asarray(a["row"], np.int64), np.asarray(b["row"], np.int64))
    np.testing.assert_array_equal(np.asarray(a["col"], np.int64), np.asarray(b["col"], np.int64))
    va = np.asarray(a["val"], np.float64)
    vb = np.asarray(b["val"], np.float64)
    if bits:
        np.testing.assert_array_equal(va.view(np.uint64), vb.view(np.uint64))
    else:
        np.testing.assert_allclose(va, vb, rtol=0, atol=atol)
