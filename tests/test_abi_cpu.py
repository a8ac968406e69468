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


def test_new_entry_points_reject_bad_arguments_on_the_host(lib):
    """The trial-step, batch and metric-dot entry points check their arguments
    before anything is enqueued (here, with no GPU, a host-side answer)."""
    from registration_b200 import _lib
    L = _lib.load()
    null = ctypes.c_void_p(0)
    # batch sizes outside [1, 4096]: no workspace, argument error
    assert L.lddmm_shoot_along_batch_f32c_workspace(100, 2, 10, 0) == 0
    assert L.lddmm_shoot_along_batch_f32c_workspace(100, 2, 10, 5000) == 0
    assert L.lddmm_shoot_along_batch_f32c_workspace(100, 2, 10, 16) > 0
    assert L.lddmm_shoot_along_batch_f32c(null, 100, 2, null, null, null, 0, 10, 0.0, 1.0, 10, 1.0, null, null, null,
                                          null, 0, null) == -1
    assert L.lddmm_dataterm_value_batch_f64_workspace(2, 0, 100, 2, 100, 100, 10, 0) == 0
    # a batch of values needs a vertex stride of at least nv * d
    assert L.lddmm_dataterm_value_batch_f64(2, 0, null, 100, 2, null, 100, null, null, 100, 1.0, 10, 1e-10, 1e-10, 3,
                                            10, null, null, 0, null) == -1
    assert b"vertex_stride" in L.lddmm_last_error()
    # metric dots: 1 to 8 directions
    ptrs = (ctypes.c_void_p * 9)()
    assert L.lddmm_metric_dots_f32c_workspace(100, 2, 10, 9) == 0
    assert L.lddmm_metric_dots_f32c(null, 100, 2, 10, null, ptrs, 9, 1.0, 10, null, null, 0, null) == -1
    assert L.lddmm_metric_dots_f32c_workspace(100, 2, 10, 2) > 0
    # too large for the single-cluster kernels: one step size per launch
    assert L.lddmm_trial_batch_size(100000, 3, 200000, 200000, 0, 1) == 1
    assert L.lddmm_trial_batch_size(256, 4, 256, 256, 0, 1) == 1
