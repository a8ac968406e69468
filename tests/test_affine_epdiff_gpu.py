"""Affine / euclidean kernel parts and landmarkEPDiff's optional outputs on
the GPU, against outputs of the reference's own code (tests/golden/
reference_golden_extra.npz, written by tests/golden/make_golden.py --extra):
Kernel.applyK / applyDiffKT with KernelSpec(affine='affine' | 'euclidean')
(kernelFunctions.py:334-367, 431-448), and landmarkEPDiff with a point set,
normals and the Jacobian (pointEvolution.py:599-658).
Tolerance: relative max-abs error <= 1e-5 (fp32c kernel sums; the affine
parts themselves are FP64) and 1e-11 (fp64)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = {"fp32c": 1e-5, "fp64": 1e-11}


@pytest.fixture(scope="module")
def extra():
    return np.load(os.path.join(HERE, "golden", "reference_golden_extra.npz"))


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_affine_kernel_parts_match_the_reference(extra, precision):
    from registration_b200 import kernelFunctions as kf
    for tag in extra["aff_cases"]:
        tag = str(tag)
        affine, kname, dd = tag.split("_")
        d = int(dd[1:])
        K = kf.Kernel(name=kname, sigma=0.4, affine=affine, w1=0.7, w2=1.3, dim=d,
                      center=list(extra["aff_center_" + tag]), precision=precision)
        x, y, a = extra["aff_x_" + tag], extra["aff_y_" + tag], extra["aff_a_" + tag]
        if "aff_k_" + tag in extra.files:
            assert rel(K.applyK(x, a), extra["aff_k_" + tag]) < TOL[precision], tag
        assert rel(K.applyK(x, a, firstVar=y), extra["aff_kf_" + tag]) < TOL[precision], tag
        if affine == "euclidean":
            got = K.applyDiffKT(x, extra["aff_a1_" + tag], extra["aff_a2_" + tag], firstVar=y)
            assert rel(got, extra["aff_dkt_" + tag]) < TOL[precision], tag
            got = K.applyDiffKT(x, extra["aff_b1_" + tag], extra["aff_b2_" + tag])
            assert rel(got, extra["aff_dkts_" + tag]) < TOL[precision], tag
        else:
            with pytest.raises(NotImplementedError):
                K.applyDiffKT(x, a[None], a[None])


def test_euclidean_self_sum_is_the_elementwise_projection(extra):
    """applyK(x, a) of a euclidean kernel: the reference's firstVar=None branch
    forms (xE * a).sum() on np.matrix objects (a matrix product, which fails for
    these shapes); the library computes the elementwise projection of its
    firstVar branch, so applyK(x, a) == applyK(x, a, firstVar=x)."""
    from registration_b200 import kernelFunctions as kf
    tag = "euclidean_gauss_d3"
    K = kf.Kernel(name="gauss", sigma=0.4, affine="euclidean", w1=0.7, w2=1.3, dim=3,
                  center=list(extra["aff_center_" + tag]), precision="fp64")
    x, a = extra["aff_x_" + tag], extra["aff_a_" + tag]
    assert rel(K.applyK(x, a), K.applyK(x, a, firstVar=x)) < 1e-13


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("kname", ["gauss", "laplacian"])
def test_epdiff_optional_outputs_match_the_reference(extra, precision, kname):
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import pointEvolution as ev
    p = "epd_%s_" % kname
    K = kf.Kernel(name=kname, sigma=float(extra[p + "sigma"]), precision=precision)
    x0, a0, T = extra[p + "x0"], extra[p + "a0"], extra[p + "xt"].shape[0] - 1
    xt, at, yt, nt, Jt = ev.landmarkEPDiff(T, x0, a0, K, withJacobian=True, withNormals=extra[p + "n0"],
                                           withPointSet=extra[p + "grid"])
    tol = TOL[precision]
    assert rel(xt, extra[p + "xt"]) < tol and rel(at, extra[p + "at"]) < tol
    assert rel(yt, extra[p + "yt"]) < tol and rel(nt, extra[p + "nt"]) < tol
    assert rel(Jt, extra[p + "Jt"]) < 10 * tol
    xt2, at2, Jt2 = ev.landmarkEPDiff(T, x0, a0, K, withJacobian=True)
    assert rel(Jt2, extra[p + "Jt_only"]) < 10 * tol
