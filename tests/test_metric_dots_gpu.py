"""Metric inner products of directions (lddmm_metric_dots_*, the dotProduct of
the matching classes) against the FP64 oracle's kernel sums:
sum_t <g2[t], K(x_t, x_t) g1[t]>.  Tolerance: fp32c 1e-5, fp64 1e-11 of
sum_t sum_k |g2[t][k]| |K g1|[t][k] (the scale of the terms that cancel)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp32c": 1e-5, "fp64": 1e-11}


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("kname,order", [("gauss", 10), ("laplacian", 3)])
@pytest.mark.parametrize("n,d,m", [(1, 2, 1), (37, 3, 2), (256, 2, 2), (700, 3, 8)])
def test_metric_dots_against_oracle(oracle_lib, precision, kname, order, n, d, m):
    import oracle
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import pointEvolution as ev
    T = 5
    rng = np.random.default_rng(100 * n + d + m)
    xt = rng.uniform(-1, 1, (T + 1, n, d))
    g1 = rng.standard_normal((T, n, d))
    g2 = [rng.standard_normal((T, n, d)) for _ in range(m - 1)] + [g1]
    K = kf.Kernel(name=kname, sigma=0.4, order=order, precision=precision)
    got = ev.metric_dots(xt, g1, g2, K).cpu().numpy()
    u = np.stack([oracle.applyk(xt[t], xt[t], g1[t], 0.4, K.order) for t in range(T)])
    for l in range(m):
        want = float((g2[l] * u).sum())
        scale = float((np.linalg.norm(g2[l], axis=2) * np.linalg.norm(u, axis=2)).sum())
        assert abs(got[l] - want) <= TOL[precision] * scale, (l, got[l], want)
    again = ev.metric_dots(xt, g1, g2, K).cpu().numpy()
    assert np.array_equal(got, again)


def test_metric_dots_arguments():
    import torch
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import pointEvolution as ev
    K = kf.Kernel(name="gauss", sigma=0.4)
    xt = torch.zeros((4, 10, 2), dtype=torch.float64, device="cuda")
    g = torch.zeros((3, 10, 2), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        ev.metric_dots(xt, g, [g] * 9, K)
    with pytest.raises(ValueError):
        ev.metric_dots(xt[:2], g, [g], K)
    assert float(ev.metric_dots(xt, g, [g], K)[0]) == 0.0
