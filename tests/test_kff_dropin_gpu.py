"""registration_b200.kernelFunctions_fort, the drop-in for py-lddmm's f2py
module kernelFunctions_fort, on the GPU.

* Replay: tests/golden/kff_calls.npz holds calls that the reference's own
  kernelFunctions.py made into kernelFunctions_fort (through Kernel.applyK /
  applyDiffKT / applyDiffKmat / applyDiffK*, landmarkHamiltonianGradient, the
  surface varifold and current gradients and the curve current gradient),
  with their positional f2py argument lists and the FP64 results.  Each is
  replayed through the drop-in: fp64 to 1e-12, fp32c to 1e-5 relative.
* Stack: the oracle's numpy restatement of the matching layers (Kernel,
  shooting, adjoint, norms, SurfaceMatching / CurveMatching, cg), which stands
  in for the reference's Python here, runs with its kernel loops routed
  through the drop-in's f2py argument lists.  In fp64 it reproduces the
  reference's recorded objective traces (1e-9 relative, or 1e-12 of obj0, the
  scale of the norms whose difference each value is).  In fp32c every kernel
  sum of the line search is FP32c, so a comparison of two trial values closer
  than their FP32c error may be decided the other way and the descent may
  branch; the fp32c check is at fixed momenta: the objective at the
  reference's final momenta within 1e-5 of obj0 of the reference's final
  value, and the gradient at the initial momenta within 1e-5 relative of
  the fp64 drop-in's (near an optimum the gradient is a small difference of
  large sums, whose FP32c error is relative to the sums).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = {"fp64": 1e-12, "fp32c": 1e-5}


@pytest.fixture(scope="module")
def kff():
    from registration_b200 import kernelFunctions_fort as m
    yield m
    m.set_precision("fp32c")


def _calls():
    d = np.load(os.path.join(HERE, "golden", "kff_calls.npz"))
    out = []
    for i in range(int(d["ncalls"])):
        args = []
        for j in range(int(d["c%d_nargs" % i])):
            a = d["c%d_a%d" % (i, j)]
            args.append(a.item() if a.ndim == 0 else a)
        out.append((str(d["c%d_name" % i]), args, d["c%d_out" % i]))
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_replays_the_reference_calls(kff, precision):
    kff.set_precision(precision)
    calls = _calls()
    assert len(calls) >= 30
    for name, args, want in calls:
        got = getattr(kff, name)(*args)
        assert isinstance(got, np.ndarray) and got.dtype == np.float64 and got.flags.f_contiguous
        assert got.shape == want.shape, name
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= TOL[precision], (name, err)


def _oracle_routed_through(kff, monkeypatch):
    """Routes the oracle's kernel loops through the drop-in's f2py argument lists."""
    import oracle

    def applyk(x, y, beta, sig, ord_):
        beta = np.asarray(beta).reshape(len(y), -1)
        return kff.applyk(x, y, beta, sig, ord_, x.shape[0], y.shape[0], x.shape[1], beta.shape[1])

    def applykdifft(x, y, a1, a2, sig, ord_):
        a1, a2 = np.asarray(a1), np.asarray(a2)
        return kff.applykdifft(x, y, a1, a2, sig, ord_, x.shape[0], y.shape[0], x.shape[1], a1.shape[2],
                               a1.shape[0])

    def applykmat(x, y, b, sig, ord_):
        return kff.applykmat(x, y, b, sig, ord_, x.shape[0], y.shape[0], x.shape[1], b.shape[2])

    def applykdiffmat(x, y, b, sig, ord_):
        return kff.applykdiffmat(x, y, b, sig, ord_, x.shape[0], y.shape[0], x.shape[1])

    for nm, fn in (("applyk", applyk), ("applykdifft", applykdifft), ("applykmat", applykmat),
                   ("applykdiffmat", applykdiffmat)):
        monkeypatch.setattr(oracle, nm, fn)


def _check_stack(kff, make, want, at_final, precision, make_far=None):
    """fp64: the whole trace; fp32c: the objective at the final momenta and the
    gradient at zero momenta.  The gradient there is the data-term gradient
    d(<S1,S1> - 2 <S1,S2>), a difference of sums whose FP32c error is relative
    to the sums: the bar is 1e-5 of the self term's gradient d<S1,S1>, the
    gradient of the same problem with the target moved out of reach of the
    kernel (make_far)."""
    if precision == "fp64":
        m = make()
        trace = []
        m.optimizeMatching(trace=trace)
        got = np.array([m.obj0] + trace)
        assert got.shape == want.shape
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12 * abs(want[0]))
        return
    kff.set_precision("fp32c")
    m = make()
    m.at = np.array(at_final, copy=True)
    m.obj = None
    obj = m.objectiveFun()
    assert abs(obj - want[-1]) <= 1e-5 * abs(want[0]), (obj, want[-1], want[0])
    # the gradient at the initial (zero) momenta: near the optimum both the data-term
    # gradient (K s1 - K s2) and the momentum gradient (2 rw a - p) are small
    # differences of large sums, whose FP32c error is relative to the sums
    grads = {}
    for prec, mk in (("fp64", make), ("fp32c", make), ("self", make_far)):
        kff.set_precision("fp64" if prec == "self" else prec)
        m = mk()
        m.obj = None
        m.objectiveFun()
        grads[prec] = m.getGradient(m.gradCoeff).diff
    g32, g64, gself = grads["fp32c"], grads["fp64"], grads["self"]
    assert np.linalg.norm(g32 - g64) <= 1e-5 * np.linalg.norm(gself), (
        np.linalg.norm(g32 - g64), np.linalg.norm(g64), np.linalg.norm(gself))


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("err", ["varifold", "current"])
def test_matching_stack_on_the_dropin_reproduces_reference_traces(kff, golden, monkeypatch, precision, err):
    from oracle import lddmm_ref as ref
    kff.set_precision(precision)
    _oracle_routed_through(kff, monkeypatch)
    f, v0, v1 = golden["sm_faces"], golden["sm_v0"], golden["sm_v1"]
    param = ref.MatchingParam(timeStep=0.2, KparDiff=ref.Kernel(name="gauss", sigma=0.4),
                              KparDist=ref.Kernel(name="gauss", sigma=0.3), sigmaError=0.5, errorType=err)
    make = lambda: ref.SurfaceMatching(ref.Surface(FV=[f, v0]), ref.Surface(FV=[f, v1]), param, maxIter=6)
    far = lambda: ref.SurfaceMatching(ref.Surface(FV=[f, v0]), ref.Surface(FV=[f, v1 + 1e3]), param, maxIter=6)
    _check_stack(kff, make, golden["sm_%s_trace" % err], golden["sm_%s_at" % err], precision, far)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_curve_matching_on_the_dropin_reproduces_reference_trace(kff, golden, monkeypatch, precision):
    from oracle import lddmm_ref as ref
    kff.set_precision(precision)
    _oracle_routed_through(kff, monkeypatch)
    param = ref.MatchingParam(timeStep=0.1, KparDiff=ref.Kernel(name="gauss", sigma=0.5),
                              KparDist=ref.Kernel(name="gauss", sigma=0.5), sigmaError=1.0, errorType="current",
                              curves=True)
    make = lambda: ref.CurveMatching(ref.Curve(pointSet=golden["cm_v0"]), ref.Curve(pointSet=golden["cm_v1"]),
                                     param, maxIter=8)
    far = lambda: ref.CurveMatching(ref.Curve(pointSet=golden["cm_v0"]), ref.Curve(pointSet=golden["cm_v1"] + 1e3),
                                    param, maxIter=8)
    _check_stack(kff, make, golden["cm_current_trace"], golden["cm_current_at"], precision, far)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_each_routine_against_the_oracle(kff, oracle_lib, precision):
    """Random inputs, size arguments given and left out, list-valued a1 / a2."""
    import oracle
    kff.set_precision(precision)
    rng = np.random.default_rng(8)
    x, y = rng.uniform(0, 1, (300, 3)), rng.uniform(0, 1, (420, 3))
    b, a1, a2 = rng.standard_normal((420, 2)), rng.standard_normal((2, 300, 3)), rng.standard_normal((2, 420, 3))
    bm, bd = rng.standard_normal((300, 420, 2)), rng.standard_normal((300, 420))
    p, q, r = (rng.standard_normal((300, 3)) for _ in range(3))
    for ordr in (10, 3):
        cases = [
            (kff.applyk(x, y, b, 0.2, ordr), oracle.applyk(x, y, b, 0.2, ordr)),
            (kff.applyk(x, y, b, 0.2, ordr, 300, 420, 3, 2), oracle.applyk(x, y, b, 0.2, ordr)),
            (kff.applykdifft(x, y, list(a1), list(a2), 0.2, ordr, 300, 420, 3, 3, 2),
             oracle.applykdifft(x, y, a1, a2, 0.2, ordr)),
            (kff.applykmat(x, y, bm, 0.2, ordr), oracle.applykmat(x, y, bm, 0.2, ordr)),
            (kff.applykdiffmat(x, y, bd, 0.2, ordr, 300, 420, 3), oracle.applykdiffmat(x, y, bd, 0.2, ordr)),
            (kff.applykdiff1(x, p, q, 0.2, ordr, 300, 3), oracle.applykdiff1(x, p, q, 0.2, ordr)),
            (kff.applykdiff2(x, p, q, 0.2, ordr), oracle.applykdiff2(x, p, q, 0.2, ordr)),
            (kff.applykdiff1and2(x, p, q, 0.2, ordr), oracle.applykdiff1and2(x, p, q, 0.2, ordr)),
            (kff.applykdiff11(x, p, q, r, 0.2, ordr), oracle.applykdiff11(x, p, q, r, 0.2, ordr)),
            (kff.applykdiff12(x, p, q, r, 0.2, ordr), oracle.applykdiff12(x, p, q, r, 0.2, ordr)),
            (kff.applykdiff11and12(x, p, q, r, 0.2, ordr, 300, 3), oracle.applykdiff11and12(x, p, q, r, 0.2, ordr)),
        ]
        for k, (got, want) in enumerate(cases):
            err = np.linalg.norm(got - want) / np.linalg.norm(want)
            assert err <= TOL[precision], (ordr, k, err)
