"""The allocation-free applyK entry point, called through the C ABI.

lddmm_applyk_f32c_noalloc serves callers that cannot allocate GPU memory (a
plug-in whose host owns all device memory, an FFI caller without a CUDA
allocator, a path where cudaMalloc would synchronise the device): they pass
inputs and the output only, and the scratch lives in a fixed 32 MiB array in the
library's static device memory.  This file is collected last so that a run
stopping at the first failure has already run every other test; it passes
both alone in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5   # the fp32c kernel-sum tolerance of the other GPU tests
SCRATCH = 32 << 20   # bytes of the static scratch


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def L():
    import torch  # noqa: F401
    from registration_b200 import _lib
    return _lib.load()


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("name,order", [("gauss", 10), ("laplacian", 3)])
def test_noalloc_matches_workspace_entry_twice(L, name, order):
    import torch
    rng = np.random.default_rng(11)
    n, m, d, dimb, sigma = 6000, 9001, 3, 3, 0.08
    x = torch.from_numpy(rng.uniform(0, 1, (n, d))).cuda()
    y = torch.from_numpy(rng.uniform(0, 1, (m, d))).cuda()
    b = torch.from_numpy(rng.standard_normal((m, dimb))).cuda()
    ref = torch.empty((n, dimb), dtype=torch.float64, device="cuda")
    wsb = L.lddmm_applyk_f32c_workspace(n, m, d, dimb)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    rc = L.lddmm_applyk_f32c(x.data_ptr(), n, y.data_ptr(), m, b.data_ptr(), d, dimb, sigma, order, ref.data_ptr(),
                             ws.data_ptr(), wsb, _stream())
    assert rc == 0, L.lddmm_last_error()
    outs = []
    for _ in range(2):   # two calls in a row share (and reuse) the static scratch
        f = torch.full((n, dimb), float("nan"), dtype=torch.float64, device="cuda")
        rc = L.lddmm_applyk_f32c_noalloc(x.data_ptr(), n, y.data_ptr(), m, b.data_ptr(), d, dimb, sigma, order,
                                         f.data_ptr(), _stream())
        assert rc == 0, L.lddmm_last_error()
        outs.append(f.cpu().numpy())
    r = ref.cpu().numpy()
    for f in outs:
        assert np.isfinite(f).all()
        assert _rel(f, r) < TOL
    np.testing.assert_array_equal(outs[0], outs[1])
    # and against the FP64 oracle directly
    import oracle
    want = oracle.applyk(x.cpu().numpy(), y.cpu().numpy(), b.cpu().numpy(), sigma, order)
    assert _rel(outs[0], want) < TOL


@pytest.mark.parametrize("name,order", [("gauss", 10), ("laplacian", 3)])
def test_noalloc_near_the_cap_matches_the_oracle(L, name, order):
    """n = m = 200,000: the workspace entry point would use more than the 32 MiB
    scratch, so the allocation-free call cuts the number of source chunks
    (another summation grouping).  Sampled target rows against the FP64 oracle,
    two calls in a row."""
    import torch
    import oracle
    rng = np.random.default_rng(12)
    n = m = 200_000
    d, dimb, sigma = 3, 3, 0.05
    assert L.lddmm_applyk_f32c_workspace(n, m, d, dimb) > SCRATCH   # the capped path is the one tested
    xh, yh, bh = rng.uniform(0, 1, (n, d)), rng.uniform(0, 1, (m, d)), rng.standard_normal((m, dimb))
    x, y, b = (torch.from_numpy(t).cuda() for t in (xh, yh, bh))
    rows = np.sort(rng.choice(n, 512, replace=False))
    want = oracle.applyk(xh[rows], yh, bh, sigma, order)
    outs = []
    for _ in range(2):
        f = torch.full((n, dimb), float("nan"), dtype=torch.float64, device="cuda")
        rc = L.lddmm_applyk_f32c_noalloc(x.data_ptr(), n, y.data_ptr(), m, b.data_ptr(), d, dimb, sigma, order,
                                         f.data_ptr(), _stream())
        assert rc == 0, L.lddmm_last_error()
        outs.append(f.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])
    assert np.isfinite(outs[0]).all()
    got = outs[0][rows]
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < TOL
    row_err = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1).max()
    assert row_err.max() < TOL


def test_noalloc_rejects_shapes_beyond_the_static_scratch(L):
    import torch
    n = m = 1 << 22   # needs far more than 32 MiB of scratch; buffers are real so nothing can read out of bounds
    x = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    b = torch.zeros((m, 3), dtype=torch.float64, device="cuda")
    f = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    rc = L.lddmm_applyk_f32c_noalloc(x.data_ptr(), n, x.data_ptr(), m, b.data_ptr(), 3, 3, 0.1, 10, f.data_ptr(),
                                     _stream())
    assert rc == -2
    assert b"static scratch" in L.lddmm_last_error()
    # beyond 2^30 points: the same argument error as the workspace entry point (no launch, no access)
    rc = L.lddmm_applyk_f32c_noalloc(x.data_ptr(), (1 << 30) + 1, x.data_ptr(), m, b.data_ptr(), 3, 3, 0.1, 10,
                                     f.data_ptr(), _stream())
    assert rc == -1 and b"2^30" in L.lddmm_last_error()
