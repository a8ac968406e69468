"""Batched trial steps: lddmm_shoot_along_batch_* and
lddmm_dataterm_value_batch_* against their one-step-size counterparts, bit
for bit, for problems that run one cluster per step size side by side (the
single-launch kernels) and for larger ones that run one step size after the
other; the batch size query; argument checks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(n, d, T, seed):
    import torch
    rng = np.random.default_rng(seed)
    x0 = torch.from_numpy(rng.uniform(-1, 1, (n, d))).cuda()
    at = torch.from_numpy(0.3 * rng.standard_normal((T, n, d))).cuda()
    dr = torch.from_numpy(0.3 * rng.standard_normal((T, n, d))).cuda()
    return x0, at, dr


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("n,d,B", [(37, 2, 16), (256, 3, 5), (512, 2, 16), (700, 3, 3), (1, 3, 1)])
def test_batched_shots_equal_single_shots(precision, n, d, B):
    import torch
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import pointEvolution as ev
    T = 7
    x0, at, dr = _problem(n, d, T, 10 * n + d)
    K = kf.Kernel(name="gauss", sigma=0.4, precision=precision)
    ladder = [0.7 / 2 ** k for k in range(B - 1)] + [3e-7] if B > 1 else [0.7]
    eps = torch.tensor(ladder, dtype=torch.float64, device="cuda")
    at_b, xt_b, e_b = ev.shoot_along_batch(x0, at, dr, eps, K, regweight=0.8)
    assert at_b.shape == (B, T, n, d) and xt_b.shape == (B, T + 1, n, d) and e_b.shape == (B,)
    for b in range(B):
        at1, xt1, e1 = ev.shoot_along(x0, at, dr, eps[b], K, regweight=0.8)
        assert torch.equal(at_b[b], at1) and torch.equal(xt_b[b], xt1), b
        assert float(e_b[b]) == float(e1), b
    # repeatable
    _, xt_c, e_c = ev.shoot_along_batch(x0, at, dr, eps, K, regweight=0.8)
    assert torch.equal(xt_b, xt_c) and torch.equal(e_b, e_c)


def _curve_shapes(n, seed):
    from registration_b200 import curves as cv
    from registration_b200 import geometry as geo
    rng = np.random.default_rng(seed)
    c, _ = geo.ellipse_curve(n, 1.0, 0.6)
    return cv.Curve(pointSet=c), cv.Curve(pointSet=c + 0.05 * rng.standard_normal(c.shape)), rng


def _surface_shapes(level, seed):
    from registration_b200 import geometry as geo
    from registration_b200 import surfaces as sf
    rng = np.random.default_rng(seed)
    v, f = geo.icosphere(level)
    vt = geo.bumped_sphere(v, f, 4, 0.3, 0.1, rng)
    return sf.Surface(FV=[f, v]), sf.Surface(FV=[f, vt]), rng


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("shape,size,err", [("curve", 256, "current"), ("curve", 300, "measure"),
                                            ("curve", 900, "current"), ("surface", 2, "varifold"),
                                            ("surface", 3, "current"), ("surface", 4, "measure")])
def test_batched_values_equal_single_values(precision, shape, size, err):
    import torch
    from registration_b200 import _dataterm as dt
    from registration_b200 import kernelFunctions as kf
    from registration_b200.device import to_dev
    S, tgt, rng = _curve_shapes(size, size) if shape == "curve" else _surface_shapes(size, size)
    K = kf.Kernel(name="gauss", sigma=0.3, precision=precision)
    v0 = to_dev(S.vertices)
    nv, d = v0.shape
    B, T = 6, 4
    # vertex sets at a batch stride larger than one set, as xt[:, -1] of batched trajectories
    xt = torch.from_numpy(0.02 * rng.standard_normal((B, T + 1, nv, d))).cuda() + v0
    dshape = S.device_shape()
    tc = to_dev(tgt.centers)
    tv = to_dev(tgt.surfel if shape == "surface" else tgt.lenel)
    e_b = dt.value_batch(err, xt[:, -1], dshape, tc, tv, K)
    for b in range(B):
        e1, _ = dt.dataterm(err, xt[b, -1].contiguous(), dshape, tc, tv, K, energy=True, grad=False)
        assert float(e_b[b]) == float(e1), b


def test_trial_batch_size_and_arguments():
    import torch
    from registration_b200 import _lib
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import pointEvolution as ev
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    # bounded by the resident clusters of both kernels (8 CTAs each at 256 points, 2 at 40) and by 24
    for shot, value in (("fp32c", "fp64"), ("fp64", "fp64"), ("fp32c", "fp32c")):
        b256 = ev.trial_batch_size(256, 2, 256, 256, shot, value)
        b40 = ev.trial_batch_size(40, 3, 80, 80, shot, value)
        assert 8 <= b256 <= min(24, 2 * sms // 8), (shot, value, b256)
        assert b256 <= b40 <= 24, (shot, value, b40)
    assert ev.trial_batch_size(700, 3, 1000, 1000) == 1
    assert ev.trial_batch_size(256, 2, 256, 4000) == 1       # the value would leave the single-cluster kernel
    x0, at, dr = _problem(20, 2, 3, 1)
    K = kf.Kernel(name="gauss", sigma=0.4)
    with pytest.raises(ValueError):
        ev.shoot_along_batch(x0, at, dr, torch.zeros((2, 2), dtype=torch.float64, device="cuda"), K)
    with pytest.raises(ValueError):
        ev.shoot_along_batch(x0, at, dr, torch.zeros(2, dtype=torch.float64, device="cuda"), K,
                             xt=torch.empty((3, 4, 20, 2), dtype=torch.float64, device="cuda"))
    eps = torch.zeros(5000, dtype=torch.float64, device="cuda")
    assert _lib.query("lddmm_shoot_along_batch_f32c_workspace", 20, 2, 3, 5000) == 0
    with pytest.raises(ValueError):
        ev.shoot_along_batch(x0, at, dr, eps, K)
