"""GPU parity of the kernel sums (applyK / applyDiffKT) against the oracle.

Tolerances (the accuracy bar of the FP32 compensated path):
  fp32c: relative error <= 1e-5 against the FP64 oracle, measured as
         ||f - f_ref||_F / ||f_ref||_F and max_k ||f_k - f_ref_k|| / max_k ||f_ref_k||;
  fp64 : the same two measures <= 1e-12.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp32c": 1e-5, "fp64": 1e-12}


def _err(f, ref):
    f = np.asarray(f).reshape(len(ref), -1)
    ref = np.asarray(ref).reshape(len(ref), -1)
    glob = np.linalg.norm(f - ref) / max(np.linalg.norm(ref), 1e-300)
    rows = np.linalg.norm(f - ref, axis=1).max() / max(np.linalg.norm(ref, axis=1).max(), 1e-300)
    return max(glob, rows)


@pytest.fixture(scope="module")
def kf():
    from registration_b200 import kernelFunctions
    return kernelFunctions


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_golden_cases_applyk_difft(golden, oracle_lib, kf, precision):
    """Every golden kernel case (gauss + laplacian 0..4, d 2/3, dimb 1/3, na 1/3,
    exact coincidences and the sub-1e-8 branch) against the reference outputs."""
    for tag in golden["kernel_cases"]:
        tag = str(tag)
        name = "gauss" if tag.startswith("gauss") else "laplacian"
        order = int(tag.split("_")[0].replace(name, ""))
        K = kf.Kernel(name=name, sigma=0.35, order=order, precision=precision)
        x, y, beta = golden["applyk_x_" + tag], golden["applyk_y_" + tag], golden["applyk_beta_" + tag]
        f = K.applyK(y, beta, firstVar=x)
        assert isinstance(f, np.ndarray) and f.dtype == np.float64 and f.shape == golden["applyk_f_" + tag].shape
        assert _err(f, golden["applyk_f_" + tag]) < TOL[precision], (tag, precision)
        for na in (1, 3):
            k = "%s_na%d" % (tag, na)
            if "difft_f_" + k in golden.files:
                fd = K.applyDiffKT(y, golden["difft_a1_" + k], golden["difft_a2_" + k], firstVar=x)
                assert _err(fd, golden["difft_f_" + k]) < TOL[precision], (k, precision)


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_golden_cases_dense_weights(golden, kf, precision):
    """Kernel.applyK(matrixWeights=True) / applyDiffKmat (kff.applykmat /
    applykdiffmat) against the reference outputs of every golden kernel case."""
    for tag in golden["kernel_cases"]:
        tag = str(tag)
        name = "gauss" if tag.startswith("gauss") else "laplacian"
        order = int(tag.split("_")[0].replace(name, ""))
        K = kf.Kernel(name=name, sigma=0.35, order=order, precision=precision)
        x, y = golden["applyk_x_" + tag], golden["applyk_y_" + tag]
        f = K.applyK(y, golden["kmat_b_" + tag], firstVar=x, matrixWeights=True)
        assert isinstance(f, np.ndarray) and f.shape == golden["kmat_f_" + tag].shape
        assert _err(f, golden["kmat_f_" + tag]) < TOL[precision], (tag, precision)
        if "kdiffmat_b_" + tag in golden.files:
            fd = K.applyDiffKmat(y, golden["kdiffmat_b_" + tag], firstVar=x)
            assert _err(fd, golden["kdiffmat_f_" + tag]) < TOL[precision], (tag, precision)


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("n,m,dimb", [(1, 1, 1), (700, 1300, 1), (1500, 900, 3)])
def test_dense_weights_random_sizes(oracle_lib, kf, precision, n, m, dimb):
    rng = np.random.default_rng(n + m + dimb)
    x = rng.uniform(0, 1, (n, 3))
    y = rng.uniform(0, 1, (m, 3))
    b = rng.standard_normal((n, m, dimb))
    for name, order, sigma in [("gauss", 10, 0.1), ("laplacian", 3, 0.1)]:
        K = kf.Kernel(name=name, sigma=sigma, order=order, precision=precision)
        f = K.applyK(y, b, firstVar=x, matrixWeights=True)
        assert _err(f, oracle_lib.applykmat(x, y, b, sigma, K.order)) < TOL[precision]
        fd = K.applyDiffKmat(y, b[:, :, 0], firstVar=x)
        assert _err(fd, oracle_lib.applykdiffmat(x, y, b[:, :, 0], sigma, K.order)) < TOL[precision]
    # self-interaction form (firstVar=None): targets = sources
    b2 = rng.standard_normal((m, m, dimb))
    K = kf.Kernel(name="gauss", sigma=0.1, precision=precision)
    assert _err(K.applyK(y, b2, matrixWeights=True), oracle_lib.applykmat(y, y, b2, 0.1, 10)) < TOL[precision]


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("name,order,sigma", [("gauss", 10, 0.05), ("laplacian", 3, 0.05), ("laplacian", 1, 0.1)])
@pytest.mark.parametrize("n,m", [(1, 1), (1000, 1), (3001, 5003), (20000, 777)])
def test_random_sizes_against_oracle(oracle_lib, kf, precision, name, order, sigma, n, m):
    rng = np.random.default_rng(n * 7 + m)
    x = rng.uniform(0, 1, (n, 3))
    y = rng.uniform(0, 1, (m, 3))
    a = rng.standard_normal((m, 3))
    K = kf.Kernel(name=name, sigma=sigma, order=order, precision=precision)
    f = K.applyK(y, a, firstVar=x)
    ref = oracle_lib.applyk(x, y, a, sigma, K.order)
    assert _err(f, ref) < TOL[precision]
    p = rng.standard_normal((n, 3))
    fd = K.applyDiffKT(y, [p], [a], firstVar=x)
    refd = oracle_lib.applykdifft(x, y, p[None], a[None], sigma, K.order)
    assert _err(fd, refd) < TOL[precision]


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_self_interaction_and_2d_and_wide_weights(oracle_lib, kf, precision):
    rng = np.random.default_rng(5)
    for d, dimb in [(2, 2), (1, 3), (3, 7), (2, 1)]:
        x = rng.uniform(-1, 1, (777, d))
        a = rng.standard_normal((777, dimb))
        K = kf.Kernel(name="gauss", sigma=0.3, precision=precision)
        f = K.applyK(x, a)
        assert _err(f, oracle_lib.applyk(x, x, a, 0.3, 10)) < TOL[precision], (d, dimb)
    # Hamiltonian covector shape: na = 3, dimb = 3 (9-wide inner product), and na = 5 (split)
    x = rng.uniform(-1, 1, (900, 3))
    for na in (3, 5):
        a1 = rng.standard_normal((na, 900, 3))
        a2 = rng.standard_normal((na, 900, 3))
        K = kf.Kernel(name="laplacian", sigma=0.4, order=3, precision=precision)
        assert _err(K.applyDiffKT(x, a1, a2), oracle_lib.applykdifft(x, x, a1, a2, 0.4, 3)) < TOL[precision]


def test_device_tensors_stay_on_device(kf):
    import torch
    x = torch.rand(500, 3, dtype=torch.float64, device="cuda")
    a = torch.randn(500, 3, dtype=torch.float64, device="cuda")
    f = kf.Kernel(name="gauss", sigma=0.2).applyK(x, a)
    assert isinstance(f, torch.Tensor) and f.is_cuda and f.shape == (500, 3)


def test_deterministic_repeat(kf):
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 1, (40000, 3))
    a = rng.standard_normal((40000, 3))
    K = kf.Kernel(name="gauss", sigma=0.05)
    f1 = K.applyK(x, a)
    f2 = K.applyK(x, a)
    np.testing.assert_array_equal(f1, f2)


def test_host_pointer_rejected_without_fault(kf):
    import ctypes
    from registration_b200 import _lib
    L = _lib.load()
    arr = (ctypes.c_double * 30)()
    rc = L.lddmm_applyk_f32c(ctypes.cast(arr, ctypes.c_void_p), 10, ctypes.cast(arr, ctypes.c_void_p), 10,
                             ctypes.cast(arr, ctypes.c_void_p), 3, 1, 1.0, 10, ctypes.cast(arr, ctypes.c_void_p),
                             ctypes.cast(arr, ctypes.c_void_p), 4096, None)
    assert rc == -1 and b"device memory" in L.lddmm_last_error() or b"CUDA pointer" in L.lddmm_last_error()


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_golden_second_derivative_loops(golden, oracle_lib, kf, precision):
    """applyDiffK / applyDiffK2 / applyDiffK1and2 / applyDDiffK11and12 (kff loops)
    against the reference's outputs, applyDDiffK11 / 12 against the restated
    loops (pinned to the reference's dense matrices on the CPU)."""
    for tag in golden["second_cases"]:
        tag = str(tag)
        name = "gauss" if tag.startswith("gauss") else "laplacian"
        order = int(tag.split("_")[0].replace(name, ""))
        x, a1, a2, p = (golden["sec_%s_%s" % (k, tag)] for k in ("x", "a1", "a2", "p"))
        K = kf.Kernel(name=name, sigma=0.4, order=order, precision=precision)
        assert _err(K.applyDiffK(x, a1, a2), golden["sec_kd1_" + tag]) < TOL[precision], tag
        assert _err(K.applyDiffK2(x, a1, a2), golden["sec_kd2_" + tag]) < TOL[precision], tag
        assert _err(K.applyDiffK1and2(x, a1, a2), golden["sec_kd12_" + tag]) < TOL[precision], tag
        if "sec_dd11_" + tag in golden.files:
            assert _err(K.applyDDiffK11and12(x, a1, a2, p), golden["sec_dd1112_" + tag]) < TOL[precision], tag
            assert _err(K.applyDDiffK11(x, a1, a2, p), oracle_lib.applykdiff11(x, a1, a2, p, 0.4, order)) \
                < TOL[precision], tag
            assert _err(K.applyDDiffK12(x, a1, a2, p), oracle_lib.applykdiff12(x, a1, a2, p, 0.4, order)) \
                < TOL[precision], tag
        else:
            with pytest.raises(ValueError):
                K.applyDDiffK11(x, a1, a2, p)


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("name,order", [("gauss", 10), ("laplacian", 3)])
def test_second_derivative_loops_random_sizes(oracle_lib, kf, precision, name, order):
    rng = np.random.default_rng(order)
    n = 3001
    x = rng.uniform(0, 1, (n, 3))
    a1, a2, p = (rng.standard_normal((n, 3)) for _ in range(3))
    K = kf.Kernel(name=name, sigma=0.1, order=order, precision=precision)
    o = K.order
    assert _err(K.applyDiffK(x, a1, a2), oracle_lib.applykdiff1(x, a1, a2, 0.1, o)) < TOL[precision]
    assert _err(K.applyDiffK2(x, a1, a2), oracle_lib.applykdiff2(x, a1, a2, 0.1, o)) < TOL[precision]
    assert _err(K.applyDiffK1and2(x, a1, a2), oracle_lib.applykdiff1and2(x, a1, a2, 0.1, o)) < TOL[precision]
    assert _err(K.applyDDiffK11(x, a1, a2, p), oracle_lib.applykdiff11(x, a1, a2, p, 0.1, o)) < TOL[precision]
    assert _err(K.applyDDiffK12(x, a1, a2, p), oracle_lib.applykdiff12(x, a1, a2, p, 0.1, o)) < TOL[precision]
    assert _err(K.applyDDiffK11and12(x, a1, a2, p),
                oracle_lib.applykdiff11and12(x, a1, a2, p, 0.1, o)) < TOL[precision]


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_empty_inputs(kf, precision):
    """No targets -> an empty result; no sources -> zeros (the f2py loops'
    results for num_nodes = 0 / num_nodes_y = 0)."""
    rng = np.random.default_rng(2)
    K = kf.Kernel(name="gauss", sigma=0.3, precision=precision)
    x = rng.uniform(0, 1, (0, 3))
    y = rng.uniform(0, 1, (17, 3))
    a = rng.standard_normal((17, 3))
    f = K.applyK(y, a, firstVar=x)
    assert f.shape == (0, 3)
    f = K.applyDiffKT(y, [np.zeros((0, 3))], [a], firstVar=x)
    assert f.shape == (0, 3)
    f = K.applyK(np.zeros((0, 3)), np.zeros((0, 2)), firstVar=y)
    assert f.shape == (17, 2) and not f.any()
    f = K.applyDiffKT(np.zeros((0, 3)), [rng.standard_normal((17, 3))], [np.zeros((0, 3))], firstVar=y)
    assert f.shape == (17, 3) and not f.any()
