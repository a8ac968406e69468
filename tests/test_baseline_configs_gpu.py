"""The benchmark configurations at their own sizes, against the FP64 oracle.

* Kernel-sum microbenchmark: N = M = 2^20 points uniform in [0,1]^3, N(0,1)
  momenta, Gaussian and order-3 Laplacian kernels of sigma 0.05, applyK and
  applyDiffKT in FP32 with compensated sums.  The oracle runs on 512 target
  rows drawn uniformly from all 2^20 (rows are independent, so the sample is
  exact for them).  Bar: relative L2 error <= 1e-5, over the sampled rows and
  for every sampled row on its own.
* Curve matching: the 256-vertex ellipse (semi-axes 1, 0.6) with 4 seeded
  Gaussian bumps (width 0.3, amplitudes N(0, 0.1^2)), Gaussian deformation
  kernel sigma 0.5, current data term sigma 0.5, T = 10, 50 cg iterations at
  most, at sigmaError 1 and at sigmaError 0.02.  The plain FP64 path must
  take the oracle's decisions and reproduce its accepted-objective trace to
  1e-9 relative (or 1e-12 of obj0, the scale of the norms whose difference
  each objective value is).
* Surface matching at its size: the subdivision-5 icosphere (10,242 vertices,
  20,480 faces) with 8 bumps, Gaussian deformation kernel sigma 0.2, varifold
  sigma 0.1, T = 10: the objective and its gradient at seeded momenta, and
  the geodesic shot, against the oracle (FP64 1e-10, FP32c 1e-5 relative).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_C2 = 1 << 20


@pytest.fixture(scope="module")
def c2_inputs():
    import torch
    rng = np.random.default_rng(20240601)
    x = rng.uniform(0, 1, (N_C2, 3))
    y = rng.uniform(0, 1, (N_C2, 3))
    a = rng.standard_normal((N_C2, 3))
    p = rng.standard_normal((N_C2, 3))
    rows = np.sort(rng.choice(N_C2, 512, replace=False))
    dev = [torch.from_numpy(t).cuda() for t in (x, y, a, p)]
    return (x, y, a, p, rows), dev


def _errors(got, want):
    glob = np.linalg.norm(got - want) / np.linalg.norm(want)
    row = (np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)).max()
    return glob, row


@pytest.mark.parametrize("name,order", [("gauss", 10), ("laplacian", 3)])
def test_kernel_sums_at_one_million_points(oracle_lib, c2_inputs, name, order):
    import oracle
    from registration_b200 import kernelFunctions as kf
    (x, y, a, p, rows), (xd, yd, ad, pd) = c2_inputs
    K = kf.Kernel(name=name, sigma=0.05, order=order, precision="fp32c")
    f = K.applyK(yd, ad, firstVar=xd)[rows.tolist()].cpu().numpy()
    g = K.applyDiffKT(yd, [pd], [ad], firstVar=xd)[rows.tolist()].cpu().numpy()
    want_f = oracle.applyk(x[rows], y, a, 0.05, K.order)
    want_g = oracle.applykdifft(x[rows], y, p[rows][None], a[None], 0.05, K.order)
    for got, want, what in ((f, want_f, "applyK"), (g, want_g, "applyDiffKT")):
        glob, row = _errors(got, want)
        assert glob <= 1e-5, (what, glob)
        assert row <= 1e-5, (what, row)


def _curve_problem():
    from registration_b200 import geometry as geo
    rng = np.random.default_rng(3)
    v, _ = geo.ellipse_curve(256, 1.0, 0.6)
    vt, _ = geo.bumped_curve(v, 4, 0.3, 0.1, rng, n_out=256)
    return v, vt


def _accepted_trace(obj):
    trace = []
    orig = obj.acceptVarTry

    def accept():
        orig()
        trace.append(float(obj.obj))

    obj.acceptVarTry = accept
    return trace


def _oracle_curve(v, vt, sig_err, iters=50):
    from oracle import lddmm_ref as ref
    param = ref.MatchingParam(timeStep=0.1, KparDiff=ref.Kernel(name="gauss", sigma=0.5),
                              KparDist=ref.Kernel(name="gauss", sigma=0.5), sigmaError=sig_err,
                              errorType="current", curves=True)
    cm = ref.CurveMatching(ref.Curve(pointSet=v), ref.Curve(pointSet=vt), param, maxIter=iters)
    trace = []
    cm.optimizeMatching(trace=trace)
    return cm, np.array([cm.obj0] + trace)


def _gpu_curve(v, vt, sig_err, precision, lsp, iters=50):
    from registration_b200 import curveMatching as CM
    from registration_b200 import curves as cv
    from registration_b200 import kernelFunctions as kf
    param = CM.CurveMatchingParam(timeStep=0.1, KparDiff=kf.Kernel(name="gauss", sigma=0.5, precision=precision),
                                  KparDist=kf.Kernel(name="gauss", sigma=0.5, precision=precision),
                                  sigmaError=sig_err, errorType="current")
    cm = CM.CurveMatching(Template=cv.Curve(pointSet=v), Target=cv.Curve(pointSet=vt), param=param, maxIter=iters,
                          saveRate=0, lineSearchPrecision=lsp)
    trace = _accepted_trace(cm)
    cm.optimizeMatching()
    return cm, np.array([cm.obj0] + trace)


@pytest.mark.parametrize("sig_err", [1.0, 0.02])
def test_curve_matching_fp64_trace_equals_oracle(oracle_lib, sig_err):
    import logging
    logging.disable(logging.INFO)
    v, vt = _curve_problem()
    rcm, want = _oracle_curve(v, vt, sig_err)
    cm, got = _gpu_curve(v, vt, sig_err, "fp64", "fp64")
    logging.disable(logging.NOTSET)
    assert got.shape == want.shape, (len(got), len(want))
    # each value is a small difference of norms of size obj0 = Norm0 / sigmaError^2
    # (1.2e4 at sigmaError 0.02): FP64 rounding lives on that scale
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12 * abs(want[0]))
    assert cm.iter == rcm.iter


@pytest.mark.parametrize("sig_err", [1.0, 0.02])
def test_curve_matching_fp32c_reaches_an_accurate_energy(oracle_lib, sig_err):
    """FP32c kernel sums with FP64 line-search values.  The reported final
    energy is the FP64 objective of the final momenta to 1e-6 relative (the
    oracle re-evaluates it); at sigmaError 1 the run takes the oracle's
    decisions and ends at its energy to 1e-6 relative.  At sigmaError 0.02
    the 50-iteration descent branches from the FP64 one once a rounding
    difference of the FP32c shots and gradients flips a line-search decision,
    so only the leading part of the trace is compared (1e-5 relative); both
    descents take the objective down by five orders of magnitude, to minima
    within a factor 1.5 of each other (a sanity bound, not the accuracy bar:
    that is the FP64 re-evaluation above)."""
    import logging
    from oracle import lddmm_ref as ref
    logging.disable(logging.INFO)
    v, vt = _curve_problem()
    rcm, want = _oracle_curve(v, vt, sig_err)
    cm, got = _gpu_curve(v, vt, sig_err, "fp32c", "fp64")
    logging.disable(logging.NOTSET)
    # the FP64 objective at the FP32c run's final momenta
    param = ref.MatchingParam(timeStep=0.1, KparDiff=ref.Kernel(name="gauss", sigma=0.5),
                              KparDist=ref.Kernel(name="gauss", sigma=0.5), sigmaError=sig_err,
                              errorType="current", curves=True)
    chk = ref.CurveMatching(ref.Curve(pointSet=v), ref.Curve(pointSet=vt), param, maxIter=0)
    chk.at = cm.at.cpu().numpy()
    chk.obj = None
    e64 = chk.objectiveFun()
    assert abs(float(cm.obj) - e64) <= 1e-6 * abs(e64), (float(cm.obj), e64)
    if sig_err == 1.0:
        assert got.shape == want.shape
        np.testing.assert_allclose(got, want, rtol=1e-6)
    else:
        lead = min(10, len(want), len(got))
        np.testing.assert_allclose(got[:lead], want[:lead], rtol=1e-5)
        assert float(cm.obj) <= 1.5 * want[-1] and want[-1] <= 1.5 * float(cm.obj)


@pytest.fixture(scope="module")
def c3_problem():
    from registration_b200 import geometry as geo
    rng = np.random.default_rng(5)
    v, f = geo.icosphere(5)
    vt = geo.bumped_sphere(v, f, 8, 0.25, 0.15, rng)
    at = 0.02 * np.random.default_rng(6).standard_normal((10, len(v), 3))
    return v, f, vt, at


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32c", 1e-5)])
def test_surface_objective_gradient_and_shot_at_full_size(oracle_lib, c3_problem, precision, tol):
    import torch
    from oracle import lddmm_ref as ref
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import pointEvolution as evol
    from registration_b200 import surfaceMatching as SM
    from registration_b200 import surfaces as sf
    v, f, vt, at = c3_problem
    assert v.shape == (10242, 3) and f.shape == (20480, 3)
    # geodesic shot
    K = kf.Kernel(name="gauss", sigma=0.2, precision=precision)
    KR = ref.Kernel(name="gauss", sigma=0.2)
    xt = evol.landmarkDirectEvolutionEuler(v, at, K)
    rxt = ref.landmarkDirectEvolutionEuler(v, at, KR)
    assert np.linalg.norm(xt[-1] - rxt[-1]) / np.linalg.norm(rxt[-1] - v) < tol
    # objective and gradient of the varifold matching problem at momenta `at`
    param = SM.SurfaceMatchingParam(timeStep=0.1, KparDiff=K,
                                    KparDist=kf.Kernel(name="gauss", sigma=0.1, precision=precision),
                                    sigmaError=0.01, errorType="varifold")
    sm = SM.SurfaceMatching(Template=sf.Surface(FV=[f, v]), Target=sf.Surface(FV=[f, vt]), param=param, maxIter=0,
                            testGradient=False, lineSearchPrecision=precision)
    sm.at = torch.from_numpy(at).cuda()
    sm.obj = None
    obj = float(sm.objectiveFun())
    g = sm.getGradient(sm.gradCoeff).diff.cpu().numpy()
    rparam = ref.MatchingParam(timeStep=0.1, KparDiff=KR, KparDist=ref.Kernel(name="gauss", sigma=0.1),
                               sigmaError=0.01, errorType="varifold")
    rparam.fun_obj0, rparam.fun_obj, rparam.fun_objGrad = (ref.varifoldNorm0_pairs, ref.varifoldNormDef_pairs,
                                                           ref.varifoldNormGradient_pairs)
    rsm = ref.SurfaceMatching(ref.Surface(FV=[f, v]), ref.Surface(FV=[f, vt]), rparam, maxIter=0)
    rsm.at = at.copy()
    rsm.obj = None
    robj = rsm.objectiveFun()
    rg = rsm.getGradient(rsm.gradCoeff).diff
    # the objective is a small difference of norms: its error is measured on the scale of Norm0 / sigmaError^2
    assert abs(obj - robj) <= tol * abs(rsm.obj0), (obj, robj, rsm.obj0)
    assert np.linalg.norm(g - rg) / np.linalg.norm(rg) < tol
