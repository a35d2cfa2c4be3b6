"""The reference's own CUDA build (oracle/refgpu/build.sh into
oracle/_ref/refgpu): the library loads without a GPU and exports the C ABI
that oracle/refgpu.py binds.  Skipped where it was not built (no reference
checkout)."""
import ctypes
import os
import re
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import refgpu  # noqa: E402


def driver_exports():
    src = open(os.path.join(ROOT, "oracle", "refgpu", "driver.cu")).read()
    body = src[src.index('extern "C" {'):]
    return sorted(set(re.findall(r"^\S.*?\b(rg_\w+)\(", body, re.M)))


def test_driver_declares_the_bound_entry_points():
    names = driver_exports()
    binding = open(os.path.join(ROOT, "oracle", "refgpu.py")).read()
    assert len(names) >= 15
    for n in names:
        assert n in binding, n


@pytest.mark.parametrize("fp64", [False, True])
def test_reference_library_loads_and_exports(fp64):
    if not refgpu.available(fp64):
        pytest.skip("oracle/_ref/refgpu is not built")
    lib = ctypes.CDLL(refgpu.LIB64 if fp64 else refgpu.LIB)
    for n in driver_exports():
        assert hasattr(lib, n), n
    assert lib.rg_real_size() == (8 if fp64 else 4)
