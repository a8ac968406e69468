"""GPU parity of shooting, the Hamiltonian adjoint, EPDiff and the divergence.

Tolerance: relative error (max-abs difference over max-abs reference) <= 1e-5
for fp32c, 1e-11 for fp64, against the reference fixtures (tests/golden) and the
FP64 oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp32c": 1e-5, "fp64": 1e-11}


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def mods():
    from registration_b200 import kernelFunctions, pointEvolution
    return kernelFunctions, pointEvolution


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("kname", ["gauss", "laplacian"])
def test_evolution_golden(golden, oracle_lib, mods, precision, kname):
    kf, ev = mods
    p = "evo_%s_" % kname
    K = kf.Kernel(name=kname, sigma=float(golden[p + "sigma"]), precision=precision)
    x0, at, px1 = golden[p + "x0"], golden[p + "at"], golden[p + "px1"]
    tol = TOL[precision]
    assert rel(ev.landmarkDirectEvolutionEuler(x0, at, K), golden[p + "xt"]) < tol
    xt2, yt, Jt = ev.landmarkDirectEvolutionEuler(x0, at, K, withJacobian=True, withPointSet=golden[p + "grid"])
    assert rel(yt, golden[p + "yt"]) < tol
    assert rel(Jt, golden[p + "Jt"]) < 10 * tol
    _, nt = ev.landmarkDirectEvolutionEuler(x0, at, K, withNormals=golden[p + "n0"])
    assert rel(nt, golden[p + "nt"]) < tol
    _, Jt4 = ev.landmarkDirectEvolutionEuler(x0, at, K, withJacobian=True)
    assert rel(Jt4, golden[p + "Jt_self"]) < 10 * tol
    pxt, xt = ev.landmarkHamiltonianCovector(x0, at, px1, K, 0.7)
    assert rel(pxt, golden[p + "pxt"]) < tol
    dat, xt6, pxt6 = ev.landmarkHamiltonianGradient(x0, at, px1, K, 0.7, getCovector=True)
    assert rel(dat, golden[p + "dat"]) < tol
    xte, ate = ev.landmarkEPDiff(at.shape[0], x0, at[0], K)
    assert rel(xte, golden[p + "xt_epdiff"]) < tol
    assert rel(ate, golden[p + "at_epdiff"]) < tol


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("kname,order,sigma", [("gauss", 10, 0.2), ("laplacian", 3, 0.25)])
@pytest.mark.parametrize("n,d,T", [(3000, 3, 10), (2500, 2, 7), (1, 3, 3), (777, 1, 4), (6000, 3, 3)])
def test_shoot_covector_against_oracle(oracle_lib, mods, precision, kname, order, sigma, n, d, T):
    from oracle import lddmm_ref as ref
    kf, ev = mods
    rng = np.random.default_rng(n + d + T)
    x0 = rng.uniform(-1, 1, (n, d))
    # momenta small enough for a smooth flow (|grad v| of order 1): with rough
    # random momenta the Euler map amplifies any rounding exponentially
    at = (0.3 * sigma ** d) * rng.standard_normal((T, n, d))
    px1 = rng.standard_normal((n, d))
    K = kf.Kernel(name=kname, sigma=sigma, order=order, precision=precision)
    KR = ref.Kernel(name=kname, sigma=sigma, order=order)
    xt, energy = ev.shoot(x0, at, K, regweight=0.9, with_energy=True)
    rxt = ref.landmarkDirectEvolutionEuler(x0, at, KR)
    assert rel(xt.cpu().numpy(), rxt) < TOL[precision]
    e_ref = sum(0.9 * (1.0 / T) * (at[t] * KR.applyK(rxt[t], at[t])).sum() for t in range(T))
    assert abs(float(energy) - e_ref) <= TOL[precision] * abs(e_ref) + 1e-300
    dat, _, pxt = ev.landmarkHamiltonianGradient(x0, at, px1, K, 0.9, getCovector=True)
    rdat, _, rpxt = ref.landmarkHamiltonianGradient(x0, at, px1, KR, 0.9, getCovector=True)
    assert rel(pxt, rpxt) < TOL[precision]
    assert rel(dat, rdat) < TOL[precision]


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_divergence_against_dense(oracle_lib, mods, precision):
    from oracle import lddmm_ref as ref
    kf, _ = mods
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, (600, 3))
    y = rng.uniform(-1, 1, (500, 3))
    a = rng.standard_normal((600, 3))
    for kname, order in (("gauss", 10), ("laplacian", 2)):
        K = kf.Kernel(name=kname, sigma=0.4, order=order, precision=precision, weight=1.5)
        KR = ref.Kernel(name=kname, sigma=0.4, order=order, weight=1.5)
        assert rel(K.applyDivergence(x, a), KR.applyDivergence(x, a)) < TOL[precision]
        assert rel(K.applyDivergence(x, a, firstVar=y), KR.applyDivergence(x, a, firstVar=y)) < TOL[precision]


def test_epdiff_converges_to_direct_shooting(mods):
    """EPDiff vs direct shooting with the EPDiff momenta (the reference logs
    this difference in surfaceMatching.endOfIteration, :394-398)."""
    kf, ev = mods
    rng = np.random.default_rng(8)
    x0 = rng.uniform(-1, 1, (400, 3))
    a0 = 0.2 * rng.standard_normal((400, 3))
    K = kf.Kernel(name="gauss", sigma=0.5)
    xte, ate = ev.landmarkEPDiff(40, x0, a0, K)
    xt = ev.landmarkDirectEvolutionEuler(x0, ate, K)
    assert rel(xt[-1], xte[-1]) < 1e-6


@pytest.mark.parametrize("kname", ["gauss", "laplacian"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32c", 1e-5)])
def test_second_order_evolution_covector_gradient_match_reference(golden, kname, precision, tol):
    """secondOrderEvolution / Hamiltonian / Covector / Gradient against the
    reference's own functions (pointEvolution.py:882-1091)."""
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import pointEvolution as evol
    p = "so_%s_" % kname
    K = kf.Kernel(name=kname, sigma=0.5, order=10 if kname == "gauss" else 3, precision=precision)
    x0, a0, rhot = golden[p + "x0"], golden[p + "a0"], golden[p + "rhot"]
    px1, pa1 = [golden[p + "px1"]], [golden[p + "pa1"]]

    def close(a, b):
        return np.abs(a - b).max() <= tol * np.abs(b).max()

    xt, at = evol.secondOrderEvolution(x0, a0, rhot, K)
    assert close(xt, golden[p + "xt"]) and close(at, golden[p + "at"])
    H = evol.secondOrderHamiltonian(xt[2], at[2], rhot[2], px1[0], pa1[0], K)
    assert abs(H - float(golden[p + "H"])) <= tol * abs(float(golden[p + "H"]))
    pxt, pat, _, _ = evol.secondOrderCovector(x0, a0, rhot, px1, pa1, K)
    assert close(pxt, golden[p + "pxt"]) and close(pat, golden[p + "pat"])
    da0, drhot, _, _ = evol.secondOrderGradient(x0, a0, rhot, px1, pa1, K)
    assert close(da0, golden[p + "da0"]) and np.array_equal(drhot, golden[p + "drhot"])
