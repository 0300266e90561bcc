"""The C-ABI library loads and exports every symbol include/bbtsvd_b200.h
declares (no GPU needed; no compute calls)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bbtsvd_b200.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bbt_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "bbt_fedsvd_run" in names and "bbt_bidiagonal_svd" in names
    from excalibur_b200 import _lib
    assert sorted(_lib.EXPORTS) == names


def test_library_exports_every_declared_symbol():
    from excalibur_b200 import _lib
    L = _lib.load()
    for name in declared():
        assert hasattr(L, name), name


def test_status_strings():
    from excalibur_b200 import _lib
    L = _lib.load()
    for s in range(7):
        assert L.bbt_status_string(s)
    assert L.bbt_status_string(3).decode() == "fewer singular values than requested"


def test_reference_cpp_api_exported():
    """The drop-in for src/bbtsvd.cpp: the reference's C++ signatures
    (Excalibur include/bbtsvd.hpp) are exported with their mangled names."""
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", os.path.join(ROOT, "excalibur_b200", "libexcalibur_b200.so")],
                         capture_output=True, text=True, check=True).stdout
    for sig in ("negative_count(int, double*, double*, double)",
                "bisection_singular_values(int, double*, double*, double, double, double, int, double*, int*)",
                "bidiagonal_bisection_twisted_svd(int, double*, double*, double*, double*, double*, int)",
                "givens_mask_cache_optimized_parallel_with_simd(unsigned long, unsigned long, unsigned long, double*, bool, bool, unsigned int)",
                "block_shift_mask(unsigned long, unsigned long, unsigned long, double*, bool, bool, unsigned int)"):
        assert sig in out, sig


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from excalibur_b200 import _lib
    L = _lib.load()
    h = C.c_void_p()
    assert L.bbt_create(C.byref(h), 0) != 0
    assert not h.value
