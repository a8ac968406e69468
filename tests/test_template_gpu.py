"""GPU parity of template estimation (surfaceTemplate.py: cg over a prior
deformation of the hyper-template and one deformation per subject) against
the objective traces recorded from the reference's own SurfaceTemplate
(tests/golden), plus the gradient identity of cg's TestGradient and the
'auto' line search.

Tolerances as for the matching problems: fp64 kernel sums, every accepted
objective within 1e-9 relative; fp32c kernel sums (the ragged launches),
within 1e-5 relative and the same number of accepted iterations.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp32c": 1e-5, "fp64": 1e-9}


def _trace(obj):
    trace = []
    orig = obj.acceptVarTry

    def accept():
        orig()
        trace.append(float(obj.obj))

    obj.acceptVarTry = accept
    return trace


def _template(golden, err, lam, precision, lsp="fp64", maxIter=5):
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import surfaceMatching as SM
    from registration_b200 import surfaceTemplate as ST
    from registration_b200 import surfaces as sf
    f, v0, subs = golden["st_faces"], golden["st_v0"], golden["st_subjects"]
    param = SM.SurfaceMatchingParam(timeStep=0.2, KparDiff=kf.Kernel(name="gauss", sigma=0.4, precision=precision),
                                    KparDist=kf.Kernel(name="gauss", sigma=0.3, precision=precision),
                                    sigmaError=0.1, errorType=err)
    return ST.SurfaceTemplate(HyperTmpl=sf.Surface(FV=[f, v0]), Targets=[sf.Surface(FV=[f, s]) for s in subs],
                              param=param, maxIter=maxIter, lambdaPrior=lam, verb=False, lineSearchPrecision=lsp)


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("err,lam", [("varifold", 1.0), ("current", 0.5)])
def test_template_trace_matches_reference(golden, precision, err, lam):
    st = _template(golden, err, lam, precision)
    trace = _trace(st)
    st.computeTemplate(testGradient=(precision == "fp32c"))
    p = "st_%s_" % err
    ref = golden[p + "trace"]
    got = np.array([st.obj0] + trace)
    assert got.shape == ref.shape, (got, ref)
    np.testing.assert_allclose(got, ref, rtol=TOL[precision])
    assert st.gradEps == pytest.approx(float(golden[p + "gradEps"]), rel=TOL[precision])
    scale = np.abs(golden[p + "atAll"]).max()
    np.testing.assert_allclose(st.atAll.cpu().numpy(), golden[p + "atAll"], rtol=0, atol=10 * TOL[precision] * scale)
    np.testing.assert_allclose(st.at.cpu().numpy(), golden[p + "at"], rtol=0,
                               atol=10 * TOL[precision] * np.abs(golden[p + "at"]).max())
    tmpl = st.getVariable().vertices
    tmpl = tmpl.cpu().numpy() if hasattr(tmpl, "cpu") else tmpl
    np.testing.assert_allclose(tmpl, golden[p + "tmpl"], rtol=0, atol=10 * TOL[precision])


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_template_gradient_identity(golden, precision):
    """d/de obj(at + e dir) = gradCoeff * dotProduct(getGradient(gradCoeff), dir)
    (the check cg's TestGradient logs, conjugateGradient.py:81-92), central
    differences along a random direction after two iterations."""
    import torch
    st = _template(golden, "varifold", 0.7, precision, maxIter=2)
    st.computeTemplate(testGradient=False)
    st.objectiveFun()
    grd = st.getGradient(st.gradCoeff)
    torch.manual_seed(3)
    d = st.randomDir()
    # Richardson-extrapolated central differences (error O(h^4)); the FP32c
    # objective carries ~1e-7 relative rounding, hence its larger step
    h = 2e-5 if precision == "fp64" else 2e-3

    def central(s):
        return (float(st.updateTry(d, -s)) - float(st.updateTry(d, s))) / (2 * s)

    fd = (4 * central(h / 2) - central(h)) / 3
    [dp] = st.dotProduct(grd, [d])
    assert dp * st.gradCoeff == pytest.approx(fd, rel=1e-7 if precision == "fp64" else 1e-4)


def test_template_auto_line_search_takes_fp64_decisions(golden):
    """'auto' (FP32c data-term values refined on demand) accepts the same steps
    as FP64 data-term values in every comparison."""
    a = _template(golden, "varifold", 1.0, "fp32c", lsp="fp64")
    ta = _trace(a)
    a.computeTemplate(testGradient=False)
    b = _template(golden, "varifold", 1.0, "fp32c", lsp="auto")
    tb = _trace(b)
    b.computeTemplate(testGradient=False)
    # same decisions: same accepted steps, so bit-identical momenta (the kernel
    # sums are the same FP32c calls) and equal final energies once 'auto'
    # refines its last value (endOptim); the recorded 'auto' values themselves
    # are FP32c data-term values (relative offset ~1e-4 here)
    assert len(ta) == len(tb)
    np.testing.assert_allclose(tb, ta, rtol=1e-3)
    assert bool((a.atAll == b.atAll).all()) and bool((a.at == b.at).all())
    assert float(b.obj) == pytest.approx(float(a.obj), rel=1e-12)


def test_template_directions_expose_reference_layout(golden):
    """Direction.all[k].diff and atAll[k] index like the reference's lists."""
    st = _template(golden, "current", 1.0, "fp32c", maxIter=1)
    st.objectiveFun()
    g = st.getGradient(st.gradCoeff)
    assert len(g.all) == st.Ntarg
    for k in range(st.Ntarg):
        assert g.all[k].diff.shape == (st.Tsize, st.npt, 3)
        assert bool((g.all[k].diff == g.stack[k]).all())
    assert st.atAll[1].shape == (st.Tsize, st.npt, 3)
