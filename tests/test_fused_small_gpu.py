"""Single-launch shooting and Hamiltonian adjoint for point sets of at most
512 points (one thread-block cluster runs all T steps), against the FP64
oracle: trajectories, deformation energy, covectors and the gradient, at
cluster sizes 1 to 8, at the edges of the per-CTA target split and on both
sides of the 512-point limit.
Tolerance as the other evolution tests: relative max-abs error <= 1e-5 for
fp32c, 1e-11 for fp64; repeated calls are bit-identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp32c": 1e-5, "fp64": 1e-11}


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("kname,order,sigma", [("gauss", 10, 0.3), ("laplacian", 3, 0.35), ("laplacian", 1, 0.35)])
@pytest.mark.parametrize("n,d", [(2, 3), (37, 2), (128, 3), (129, 3), (256, 2), (511, 3), (512, 2), (640, 3)])
def test_fused_shoot_and_adjoint_against_oracle(oracle_lib, precision, kname, order, sigma, n, d):
    import torch
    from oracle import lddmm_ref as ref
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import pointEvolution as ev
    T = 10
    rng = np.random.default_rng(1000 * n + d + order)
    x0 = rng.uniform(-1, 1, (n, d))
    at = (0.3 * sigma ** d) * rng.standard_normal((T, n, d))
    px1 = rng.standard_normal((n, d))
    K = kf.Kernel(name=kname, sigma=sigma, order=order, precision=precision)
    KR = ref.Kernel(name=kname, sigma=sigma, order=order)
    xt, energy = ev.shoot(x0, at, K, regweight=0.8, with_energy=True)
    xt2, energy2 = ev.shoot(x0, at, K, regweight=0.8, with_energy=True)
    assert torch.equal(xt, xt2) and float(energy) == float(energy2)
    rxt = ref.landmarkDirectEvolutionEuler(x0, at, KR)
    assert rel(xt.cpu().numpy(), rxt) < TOL[precision]
    e_ref = sum(0.8 * (1.0 / T) * (at[t] * KR.applyK(rxt[t], at[t])).sum() for t in range(T))
    assert abs(float(energy) - e_ref) <= TOL[precision] * abs(e_ref)
    pxt, dat = ev.covector(xt, at, px1, K, 0.8)
    pxt2, dat2 = ev.covector(xt, at, px1, K, 0.8)
    assert torch.equal(pxt, pxt2) and torch.equal(dat, dat2)
    rdat, _, rpxt = ref.landmarkHamiltonianGradient(x0, at, px1, KR, 0.8, getCovector=True)
    assert rel(pxt.cpu().numpy(), rpxt) < TOL[precision]
    assert rel(dat.cpu().numpy(), rdat) < TOL[precision]


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_fused_shot_without_energy_and_with_explicit_step(oracle_lib, precision):
    """energy = NULL and an explicit dt (a segment of a longer shot)."""
    from oracle import lddmm_ref as ref
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import pointEvolution as ev
    rng = np.random.default_rng(5)
    n, d, T = 300, 3, 4
    x0 = rng.uniform(-1, 1, (n, d))
    at = 0.01 * rng.standard_normal((T, n, d))
    K = kf.Kernel(name="gauss", sigma=0.3, precision=precision)
    xt, e = ev.shoot(x0, at, K, dt=0.05)
    assert e is None
    want = np.zeros((T + 1, n, d))
    want[0] = x0
    KR = ref.Kernel(name="gauss", sigma=0.3)
    for t in range(T):
        want[t + 1] = want[t] + 0.05 * KR.applyK(want[t], at[t])
    assert rel(xt.cpu().numpy(), want) < TOL[precision]
