"""The restated introsort (detnqs_b200/csrc/refsort.cuh), which puts tied
heat-bath weights in the reference's order on the GPU, against libstdc++'s
std::sort -- the implementation of the reference's
std::ranges::sort(row, std::greater{}, &Entry::w) (hb_table.cpp:133) -- and
its heapsort fallback against std::partial_sort, compiled for the host from
the same header (tests/refsort_check.cpp)."""

from __future__ import annotations

import os
import subprocess

from conftest import ROOT


def test_restated_sort_equals_std_sort(tmp_path):
    exe = str(tmp_path / "refsort_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-o", exe,
                    os.path.join(ROOT, "tests", "refsort_check.cpp")], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    assert out.startswith("ok "), out
