"""The C-ABI library builds, loads and exports every declared symbol
(CPU-only: no kernel is launched)."""

import ctypes
import os
import re

import pytest

from cloudfem_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cfem.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"CFEM_API\s+[\w\s\*]*?\b(cfem_\w+)\s*\(",
                                 text)))


def test_header_declares_api():
    syms = declared_symbols()
    assert "cfem_pcg_solve" in syms and "cfem_assemble" in syms
    assert len(syms) >= 19


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_native.LIB_PATH):
        pytest.skip("libcfem.so not built")
    lib = ctypes.CDLL(_native.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"missing exports: {missing}"


def test_binding_covers_header():
    bound = {name for name, _, _ in _native.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_library_loads_and_reports_version():
    if not os.path.exists(_native.LIB_PATH):
        pytest.skip("libcfem.so not built")
    lib = _native.load_library()
    assert lib.cfem_version() >= 10000
    assert isinstance(lib.cfem_last_error(), bytes)


def test_struct_layouts_match_header():
    # cfem_coef: ptr, double, int32, int32
    assert ctypes.sizeof(_native.Coef) == 24
    # cfem_linsys: 8+4+4 + 7 ptrs + 8 + 4 + 4
    assert ctypes.sizeof(_native.LinSys) == 16 + 7 * 8 + 16 + 8 + 8 + 8
    assert ctypes.sizeof(_native.SolveStats) == 56
    # cfem_mixed_job: int64, int32, int32, 4 pointers
    assert ctypes.sizeof(_native.MixedJob) == 8 + 4 + 4 + 4 * 8
