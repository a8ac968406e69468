"""Single-launch data-term values and gradients (shapes of at most 512 cells: one
thread-block cluster computes the cell geometry, the packing frame, the sums
and the energy) against the FP64 oracle, for the three norms on surfaces and
the two on curves, NormDef and Norm0, on both sides of the 512-cell limit.
Tolerance: values fp32c 1e-5, fp64 1e-12, of the target's Norm0 (the scale of
the norms whose difference NormDef is); gradients fp32c 1e-5, fp64 1e-11, of
the self term's gradient (the scale of the sums they are differences of)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp32c": 1e-5, "fp64": 1e-12}
GTOL = {"fp32c": 1e-5, "fp64": 1e-11}


def _surface(nf_target, seed):
    from registration_b200 import geometry as geo
    rng = np.random.default_rng(seed)
    lvl = 1
    while 20 * 4 ** lvl < nf_target:
        lvl += 1
    v, f = geo.icosphere(lvl)
    if len(f) > nf_target:
        v, f = geo.decimate(v, f, nf_target // 2 + 2, rng)
    vt = geo.bumped_sphere(v, f, 4, 0.3, 0.1, rng)
    vd = v + 0.02 * rng.standard_normal(v.shape)
    return v, f, vt, vd


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("err", ["current", "measure", "varifold"])
@pytest.mark.parametrize("nf", [80, 320, 500, 640])
def test_surface_values_against_oracle(oracle_lib, precision, err, nf):
    from oracle import lddmm_ref as ref
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import surfaces as sf
    v, f, vt, vd = _surface(nf, nf)
    K = kf.Kernel(name="gauss", sigma=0.2, precision=precision)
    KR = ref.Kernel(name="gauss", sigma=0.2)
    a, b = sf.Surface(FV=[f, vd]), sf.Surface(FV=[f, vt])
    ra, rb = ref.Surface(FV=[f, vd]), ref.Surface(FV=[f, vt])
    n0 = getattr(ref, err + "Norm0")(rb, KR)
    assert abs(getattr(sf, err + "Norm0")(b, K) - n0) <= TOL[precision] * abs(n0)
    e = getattr(sf, err + "NormDef")(a, b, K)
    assert abs(e - getattr(ref, err + "NormDef")(ra, rb, KR)) <= TOL[precision] * abs(n0)
    assert e == getattr(sf, err + "NormDef")(a, b, K)   # repeatable


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("err", ["current", "measure"])
@pytest.mark.parametrize("n,d,kname", [(256, 2, "gauss"), (256, 2, "laplacian"), (500, 3, "gauss"), (600, 2, "gauss"),
                                       (7, 2, "laplacian")])
def test_curve_values_against_oracle(oracle_lib, precision, err, n, d, kname):
    from oracle import lddmm_ref as ref
    from registration_b200 import curves as cv
    from registration_b200 import geometry as geo
    from registration_b200 import kernelFunctions as kf
    rng = np.random.default_rng(n + d)
    c, _ = geo.ellipse_curve(n, 1.0, 0.6)
    if d == 3:
        c = np.concatenate([c, 0.1 * np.sin(np.arange(n))[:, None]], axis=1)
    ct = c + 0.05 * rng.standard_normal(c.shape)
    cd = c + 0.02 * rng.standard_normal(c.shape)
    K = kf.Kernel(name=kname, sigma=0.5, order=3, precision=precision)
    KR = ref.Kernel(name=kname, sigma=0.5, order=3)
    a, b = cv.Curve(pointSet=cd), cv.Curve(pointSet=ct)
    ra, rb = ref.Curve(pointSet=cd), ref.Curve(pointSet=ct)
    n0 = getattr(ref, "curve_" + err + "Norm0")(rb, KR)
    assert abs(getattr(cv, err + "Norm0")(b, K) - n0) <= TOL[precision] * abs(n0)
    e_ref = getattr(ref, "curve_" + err + "NormDef")(ra, rb, KR)
    assert abs(getattr(cv, err + "NormDef")(a, b, K) - e_ref) <= TOL[precision] * abs(n0)


def _self_scale(ref_mod, shape_cls, fvD, grad_fn, K, vec_attr, **kw):
    """max |gradient of |S1|^2| by the oracle against a target with zero cell
    vectors: the scale of the sums whose difference the gradient is."""
    tgt = shape_cls(**kw)
    setattr(tgt, vec_attr, np.zeros_like(getattr(tgt, vec_attr)))
    return np.abs(grad_fn(fvD, tgt, K)).max()


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("err", ["current", "measure", "varifold"])
@pytest.mark.parametrize("nf", [80, 320, 500, 640])
@pytest.mark.parametrize("kname", ["gauss", "laplacian"])
def test_surface_gradients_against_oracle(oracle_lib, precision, err, nf, kname):
    """NormGradient of small surfaces (one cluster launch up to 512 cells, the
    general path above): the largest error at most TOL of the self term's
    gradient (or of the gradient itself, when larger)."""
    from oracle import lddmm_ref as ref
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import surfaces as sf
    v, f, vt, vd = _surface(nf, nf + 1)
    K = kf.Kernel(name=kname, sigma=0.2, order=3, precision=precision)
    KR = ref.Kernel(name=kname, sigma=0.2, order=3)
    g = getattr(sf, err + "NormGradient")(sf.Surface(FV=[f, vd]), sf.Surface(FV=[f, vt]), K)
    rg = getattr(ref, err + "NormGradient")(ref.Surface(FV=[f, vd]), ref.Surface(FV=[f, vt]), KR)
    G = _self_scale(ref, ref.Surface, ref.Surface(FV=[f, vd]), getattr(ref, err + "NormGradient"), KR, "surfel",
                    FV=[f, vt])
    assert g.shape == rg.shape
    assert np.abs(g - rg).max() <= GTOL[precision] * max(G, np.abs(rg).max())
    assert np.array_equal(g, getattr(sf, err + "NormGradient")(sf.Surface(FV=[f, vd]), sf.Surface(FV=[f, vt]), K))


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("err", ["current", "measure"])
@pytest.mark.parametrize("n,d,kname", [(256, 2, "gauss"), (256, 2, "laplacian"), (300, 3, "gauss"), (600, 2, "gauss"),
                                       (7, 2, "laplacian")])
def test_curve_gradients_against_oracle(oracle_lib, precision, err, n, d, kname):
    from oracle import lddmm_ref as ref
    from registration_b200 import curves as cv
    from registration_b200 import geometry as geo
    from registration_b200 import kernelFunctions as kf
    rng = np.random.default_rng(10 * n + d)
    c, _ = geo.ellipse_curve(n, 1.0, 0.6)
    if d == 3:
        c = np.concatenate([c, 0.1 * np.sin(np.arange(n))[:, None]], axis=1)
    ct = c + 0.05 * rng.standard_normal(c.shape)
    cd = c + 0.02 * rng.standard_normal(c.shape)
    K = kf.Kernel(name=kname, sigma=0.5, order=3, precision=precision)
    KR = ref.Kernel(name=kname, sigma=0.5, order=3)
    g = getattr(cv, err + "NormGradient")(cv.Curve(pointSet=cd), cv.Curve(pointSet=ct), K)
    rfn = getattr(ref, "curve_" + err + "NormGradient")
    rg = rfn(ref.Curve(pointSet=cd), ref.Curve(pointSet=ct), KR)
    G = _self_scale(ref, ref.Curve, ref.Curve(pointSet=cd), rfn, KR, "lenel", pointSet=ct)
    assert g.shape == rg.shape
    assert np.abs(g - rg).max() <= GTOL[precision] * max(G, np.abs(rg).max())
