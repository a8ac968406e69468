"""GPU parity of the surface / curve data-attachment norms and gradients.

Against the reference fixtures (tests/golden) and the FP64 oracle.
Tolerance: fp32c 1e-5, fp64 1e-11, relative to the magnitude of the summed
terms: values against |Norm0| of the target; gradients against the largest
entry of the gradient of |S1|^2 alone (the target term has the same size).
A gradient of |S1 - S2|^2 between nearby shapes is a small difference of two
such sums, so its own magnitude is not the scale of the FP32 rounding.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp32c": 1e-5, "fp64": 1e-11}


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def self_scale(ref_mod, shape_cls, fvD, grad_fn, K, vec_attr, **kw):
    """max |gradient of |S1|^2| computed by the oracle against a null target."""
    tgt = shape_cls(**kw)
    setattr(tgt, vec_attr, np.zeros_like(getattr(tgt, vec_attr)))
    return np.abs(grad_fn(fvD, tgt, K)).max()


@pytest.fixture(scope="module")
def mods():
    from registration_b200 import curves, kernelFunctions, surfaces
    return kernelFunctions, surfaces, curves


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("kname,sig", [("gauss", 0.4), ("laplacian", 0.5)])
@pytest.mark.parametrize("err", ["current", "measure", "varifold"])
def test_surface_norms_golden(golden, mods, precision, kname, sig, err):
    kf, sf, _ = mods
    f = golden["surf_faces"]
    fv1 = sf.Surface(FV=[f, golden["surf_vtgt"]])
    fvD = sf.Surface(FV=[f, golden["surf_vdef"]])
    np.testing.assert_array_equal(fvD.centers, golden["surf_centers"])
    np.testing.assert_array_equal(fvD.surfel, golden["surf_surfel"])
    K = kf.Kernel(name=kname, sigma=sig, precision=precision)
    p = "surf_%s_%s_" % (err, kname)
    n0 = getattr(sf, err + "Norm0")(fv1, K)
    scale = abs(float(golden[p + "norm0"]))
    assert abs(n0 - golden[p + "norm0"]) <= TOL[precision] * scale
    nd = getattr(sf, err + "NormDef")(fvD, fv1, K)
    assert abs(nd - golden[p + "normdef"]) <= TOL[precision] * max(scale, abs(float(golden[p + "normdef"])))
    g = getattr(sf, err + "NormGradient")(fvD, fv1, K)
    from oracle import lddmm_ref as ref
    KR = ref.Kernel(name=kname, sigma=sig)
    G = self_scale(ref, ref.Surface, ref.Surface(FV=[f, golden["surf_vdef"]]), getattr(ref, err + "NormGradient"),
                   KR, "surfel", FV=[f, golden["surf_vtgt"]])
    assert np.abs(g - golden[p + "grad"]).max() < TOL[precision] * max(G, np.abs(golden[p + "grad"]).max())


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("kname", ["gauss", "laplacian"])
@pytest.mark.parametrize("err", ["current", "measure"])
def test_curve_norms_golden(golden, mods, precision, kname, err):
    kf, _, cv = mods
    fv1 = cv.Curve(pointSet=golden["curve_vtgt"])
    fvD = cv.Curve(pointSet=golden["curve_vdef"])
    K = kf.Kernel(name=kname, sigma=0.5, precision=precision)
    p = "curve_%s_%s_" % (err, kname)
    scale = abs(float(golden[p + "norm0"]))
    assert abs(getattr(cv, err + "Norm0")(fv1, K) - golden[p + "norm0"]) <= TOL[precision] * scale
    assert abs(getattr(cv, err + "NormDef")(fvD, fv1, K) - golden[p + "normdef"]) <= TOL[precision] * scale
    from oracle import lddmm_ref as ref
    KR = ref.Kernel(name=kname, sigma=0.5)
    G = self_scale(ref, ref.Curve, ref.Curve(pointSet=golden["curve_vdef"]), getattr(ref, "curve_" + err +
                   "NormGradient"), KR, "lenel", pointSet=golden["curve_vtgt"])
    g = getattr(cv, err + "NormGradient")(fvD, fv1, K)
    assert np.abs(g - golden[p + "grad"]).max() < TOL[precision] * max(G, np.abs(golden[p + "grad"]).max())


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("err", ["current", "measure", "varifold"])
@pytest.mark.parametrize("subdiv", [3, 4])
def test_surface_norms_larger_mesh_against_oracle(oracle_lib, mods, precision, err, subdiv):
    """Subdivision-3 / 4 icospheres (1280 / 5120 faces: the small and the large
    tile shapes of the sweeps) vs the oracle's formulas."""
    from oracle import lddmm_ref as ref
    from registration_b200 import geometry as geo
    kf, sf, _ = mods
    rng = np.random.default_rng(17)
    v, f = geo.icosphere(subdiv)
    vt = geo.bumped_sphere(v, f, 8, 0.25, 0.15, rng)
    vd = v + 0.02 * rng.standard_normal(v.shape)
    K = kf.Kernel(name="gauss", sigma=0.1, precision=precision)
    KR = ref.Kernel(name="gauss", sigma=0.1)
    a, b = sf.Surface(FV=[f, vd]), sf.Surface(FV=[f, vt])
    ra, rb = ref.Surface(FV=[f, vd]), ref.Surface(FV=[f, vt])
    e_ref = getattr(ref, err + "NormDef")(ra, rb, KR)
    n0 = getattr(ref, err + "Norm0")(rb, KR)
    assert abs(getattr(sf, err + "NormDef")(a, b, K) - e_ref) <= TOL[precision] * abs(n0)
    assert rel(getattr(sf, err + "NormGradient")(a, b, K), getattr(ref, err + "NormGradient")(ra, rb, KR)) \
        < TOL[precision]


def test_open_curve_keeps_reference_faces(mods):
    _, _, cv = mods
    c = cv.Curve(pointSet=np.random.default_rng(0).standard_normal((5, 2)), isOpen=True)
    assert c.faces.tolist() == [[0, 1], [1, 2], [2, 3], [3, 4], [0, 0]]
