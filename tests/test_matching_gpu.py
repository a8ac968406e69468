"""GPU parity of the full matching problems (cg + shooting + adjoint + data
terms) against the objective traces recorded from the reference's own
SurfaceMatching / CurveMatching / cg (tests/golden).

Tolerance: fp64 path, every accepted objective within 1e-9 relative; fp32c
path (FP32 shooting / adjoint / data-term gradients, FP64 line-search values),
the same number of accepted iterations, every objective within 1e-5 relative
and the final objective within 1e-6 absolute -- the reference's own absolute
convergence threshold on the objective (conjugateGradient.py:186).
"""
import logging

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp32c": 1e-5, "fp64": 1e-9}


def check_trace(got, ref, precision):
    assert got.shape == ref.shape, (got, ref)
    np.testing.assert_allclose(got, ref, rtol=TOL[precision])
    assert abs(got[-1] - ref[-1]) <= (1e-6 if precision == "fp32c" else 1e-9 * abs(ref[-1]))


def _trace(obj):
    trace = []
    orig = obj.acceptVarTry

    def accept():
        orig()
        trace.append(float(obj.obj))

    obj.acceptVarTry = accept
    return trace


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("err", ["varifold", "current", "measure"])
def test_surface_matching_trace(golden, precision, err):
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import surfaceMatching as SM
    from registration_b200 import surfaces as sf
    f, v0, v1 = golden["sm_faces"], golden["sm_v0"], golden["sm_v1"]
    param = SM.SurfaceMatchingParam(timeStep=0.2, KparDiff=kf.Kernel(name="gauss", sigma=0.4, precision=precision),
                                    KparDist=kf.Kernel(name="gauss", sigma=0.3, precision=precision),
                                    sigmaError=0.5, errorType=err)
    sm = SM.SurfaceMatching(Template=sf.Surface(FV=[f, v0]), Target=sf.Surface(FV=[f, v1]), param=param, maxIter=6,
                            testGradient=False)
    trace = _trace(sm)
    sm.optimizeMatching()
    check_trace(np.array([sm.obj0] + trace), golden["sm_%s_trace" % err], precision)
    np.testing.assert_allclose(sm.at.cpu().numpy(), golden["sm_%s_at" % err], rtol=0,
                               atol=10 * TOL[precision] * np.abs(golden["sm_%s_at" % err]).max())


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("err", ["current", "measure"])
def test_curve_matching_trace(golden, precision, err):
    from registration_b200 import curveMatching as CM
    from registration_b200 import curves as cv
    from registration_b200 import kernelFunctions as kf
    param = CM.CurveMatchingParam(timeStep=0.1, KparDiff=kf.Kernel(name="gauss", sigma=0.5, precision=precision),
                                  KparDist=kf.Kernel(name="gauss", sigma=0.5, precision=precision), sigmaError=1.0,
                                  errorType=err)
    cm = CM.CurveMatching(Template=cv.Curve(pointSet=golden["cm_v0"]), Target=cv.Curve(pointSet=golden["cm_v1"]),
                          param=param, maxIter=8, saveRate=0)
    trace = _trace(cm)
    cm.optimizeMatching()
    check_trace(np.array([cm.obj0] + trace), golden["cm_%s_trace" % err], precision)


def test_user_plugged_data_term_is_honoured(golden):
    """SurfaceMatchingParam's fun_obj triple is a plug-in point: a user triple is called."""
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import surfaceMatching as SM
    from registration_b200 import surfaces as sf
    calls = {"n": 0}

    def my_def(a, b, K):
        calls["n"] += 1
        return sf.currentNormDef(a, b, K)

    f, v0, v1 = golden["sm_faces"], golden["sm_v0"], golden["sm_v1"]
    param = SM.SurfaceMatchingParam(timeStep=0.2, KparDiff=kf.Kernel(name="gauss", sigma=0.4),
                                    KparDist=kf.Kernel(name="gauss", sigma=0.3), sigmaError=0.5, errorType="current")
    param.fun_obj = my_def
    sm = SM.SurfaceMatching(Template=sf.Surface(FV=[f, v0]), Target=sf.Surface(FV=[f, v1]), param=param, maxIter=2,
                            testGradient=True)
    logging.disable(logging.INFO)
    sm.optimizeMatching()
    logging.disable(logging.NOTSET)
    assert calls["n"] > 0


def test_matching_from_mesh_files(golden, tmp_path):
    """fileTempl / fileTarg (surfaceMatching.py:83-97) read .byu / .vtk files."""
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import meshio
    from registration_b200 import surfaceMatching as SM
    from registration_b200 import surfaces as sf
    f, v0, v1 = golden["sm_faces"], golden["sm_v0"], golden["sm_v1"]
    p0, p1 = str(tmp_path / "t.byu"), str(tmp_path / "s.vtk")
    sf.Surface(FV=[f, v0]).savebyu(p0)
    sf.Surface(FV=[f, v1]).saveVTK(p1)
    param = SM.SurfaceMatchingParam(timeStep=0.2, KparDiff=kf.Kernel(name="gauss", sigma=0.4),
                                    KparDist=kf.Kernel(name="gauss", sigma=0.3), sigmaError=0.5, errorType="varifold")
    a = SM.SurfaceMatching(fileTempl=p0, fileTarg=p1, param=param, maxIter=2, testGradient=False)
    va, fa = meshio.read_byu(p0)
    vb, fb = meshio.read_vtk(p1)
    b = SM.SurfaceMatching(Template=sf.Surface(FV=[fa, va]), Target=sf.Surface(FV=[fb, vb]), param=param, maxIter=2,
                           testGradient=False)
    a.optimizeMatching()
    b.optimizeMatching()
    assert float(a.obj) == float(b.obj)
    assert bool((a.at == b.at).all())


@pytest.mark.parametrize("case", ["surface-auto", "surface-fp64", "curve-fp32c"])
def test_graphed_trials_equal_eager_trials(golden, case):
    """cudaGraphs=True replays the same kernels on the same inputs: the traces
    and the momenta are bit-identical to the eager path.  On these small shapes
    the graph evaluates the line search's step sizes in batches, so it takes
    fewer launches than there are trial steps."""
    from registration_b200 import curveMatching as CM
    from registration_b200 import curves as cv
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import surfaceMatching as SM
    from registration_b200 import surfaces as sf
    import torch
    runs = []
    for graphs in (False, True):
        torch.manual_seed(11)     # the same TestGradient directions in both runs
        if case.startswith("surface"):
            prec = "fp64" if case.endswith("fp64") else "fp32c"
            f, v0, v1 = golden["sm_faces"], golden["sm_v0"], golden["sm_v1"]
            param = SM.SurfaceMatchingParam(timeStep=0.2, KparDiff=kf.Kernel(name="gauss", sigma=0.4, precision=prec),
                                            KparDist=kf.Kernel(name="gauss", sigma=0.3, precision=prec),
                                            sigmaError=0.5, errorType="varifold")
            m = SM.SurfaceMatching(Template=sf.Surface(FV=[f, v0]), Target=sf.Surface(FV=[f, v1]), param=param,
                                   maxIter=6, testGradient=True, lineSearchPrecision="auto" if prec == "fp32c" else "fp64",
                                   cudaGraphs=graphs)
        else:
            param = CM.CurveMatchingParam(timeStep=0.1, KparDiff=kf.Kernel(name="gauss", sigma=0.5),
                                          KparDist=kf.Kernel(name="gauss", sigma=0.5), sigmaError=1.0,
                                          errorType="current")
            m = CM.CurveMatching(Template=cv.Curve(pointSet=golden["cm_v0"]), Target=cv.Curve(pointSet=golden["cm_v1"]),
                                 param=param, maxIter=8, saveRate=0, lineSearchPrecision="fp32c", cudaGraphs=graphs)
        trace = _trace(m)
        m.optimizeMatching()
        runs.append((trace, m.at.clone(), float(m.obj), dict(m.calls)))
    (t0, a0, o0, c0), (t1, a1, o1, c1) = runs
    batches = c1.pop("trial_batches")
    assert t0 == t1 and o0 == o1 and c0 == c1
    assert bool((a0 == a1).all())
    assert "trial_batches" not in c0 and 0 < batches < c1["updateTry"] / 2, (batches, c1)
