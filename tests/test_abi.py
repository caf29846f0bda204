"""The C-ABI library loads and exports every entry point include/*.h
declares (no compute calls: runs without a GPU)."""

from __future__ import annotations

import ctypes
import glob
import os
import re

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(dnq_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_header_declares_entry_points():
    d = _declared()
    assert "dnq_build" in d and "dnq_ham_spmv" in d and len(d) >= 20


def test_library_exports_every_declared_symbol():
    from detnqs_b200 import native
    lib = ctypes.CDLL(native.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(native.EXPORTS) <= set(_declared())


def test_library_resolves_every_symbol_at_load():
    """Immediate binding: an internal function referenced across files but
    never defined (e.g. left in an unnamed namespace) fails here, on CPU."""
    import os
    from detnqs_b200 import native
    ctypes.CDLL(native.LIB_PATH, mode=os.RTLD_NOW)


def test_version_and_error_string_without_gpu():
    from detnqs_b200 import native
    assert native.lib.dnq_version() >= 100
    assert isinstance(native.lib.dnq_last_error(), bytes)
