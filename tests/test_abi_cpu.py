"""CPU tests of the C ABI library: it loads, exports every symbol that
include/lddmm_b200.h declares, and the Python binding covers all of them.
No compute call is made (there is no GPU here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lddmm_b200.h")


def header_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"LDDMM_API\s+[\w\s\*]*?\b(lddmm_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from registration_b200 import _lib, build
    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return ctypes.CDLL(_lib.LIB_PATH)


def test_header_declares_symbols():
    syms = header_symbols()
    assert "lddmm_applyk_f32c" in syms and "lddmm_applykdifft_f64" in syms
    assert len(syms) >= 10


def test_library_exports_every_header_symbol(lib):
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    from registration_b200 import _lib
    assert set(header_symbols()) == set(_lib.SIGNATURES), set(header_symbols()) ^ set(_lib.SIGNATURES)


def test_workspace_queries_without_gpu(lib):
    from registration_b200 import _lib
    L = _lib.load()
    assert L.lddmm_abi_version() >= 1
    assert L.lddmm_applyk_f32c_workspace(1000, 2000, 3, 3) > 0
    assert L.lddmm_applyk_f64_workspace(1000, 2000, 3, 3) > 0
    assert L.lddmm_applykdifft_f32c_workspace(1000, 2000, 3, 3, 3) > 0
    # invalid shapes -> 0
    assert L.lddmm_applyk_f32c_workspace(10, 10, 4, 3) == 0
    assert L.lddmm_applykdifft_f32c_workspace(10, 10, 5, 3, 3) == 0


def test_invalid_arguments_are_rejected_before_any_launch(lib):
    from registration_b200 import _lib
    L = _lib.load()
    null = ctypes.c_void_p(0)
    # d = 4 unsupported, sigma <= 0, order-0 derivative: all rejected on the host
    assert L.lddmm_applyk_f32c(null, 10, null, 10, null, 4, 3, 1.0, 10, null, null, 0, null) == -1
    assert L.lddmm_applyk_f32c(null, 10, null, 10, null, 3, 3, 0.0, 10, null, null, 0, null) == -1
    assert L.lddmm_applykdifft_f32c(null, 10, null, 10, null, null, 1, 3, 3, 1.0, 0, null, null, 0, null) == -1
    assert b"not differentiable" in L.lddmm_last_error()
