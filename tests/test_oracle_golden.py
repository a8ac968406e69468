"""CPU tests: the oracle against the fixtures produced by running the reference.

tests/golden/make_golden.py ran the reference's own Python modules (Kernel,
pointEvolution, surfaces, curves, surfaceMatching, curveMatching, cg) on top
of the restated Fortran loops, plus the reference's dense numpy kernel
matrices.  These tests pin:
  * the restated loops against the reference's dense kernel matrices;
  * the oracle's numpy transliteration against the reference's Python.
"""
import numpy as np
import pytest

from oracle import lddmm_ref as ref


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def test_loops_match_reference_dense_matrices(golden, oracle_lib):
    """kff loops (exact-rational mode) vs kernelMatrixGauss/Laplacian @ beta."""
    for tag in golden["kernel_cases"]:
        tag = str(tag)
        dense = golden["applyk_dense_" + tag]
        tol = 1e-13 if "laplacian0" not in tag else 2e-9   # order 0: the 1e-8 zero-distance branch
        assert _rel(golden["applyk_exact_" + tag], dense) < tol, tag
        # float32 default-real literals of the Fortran tables move the Laplacian by ~1e-8
        assert _rel(golden["applyk_f_" + tag], dense) < 5e-8, tag
        for na in (1, 3):
            k = "%s_na%d" % (tag, na)
            if "difft_f_" + k in golden.files:
                assert _rel(golden["difft_exact_" + k], golden["difft_dense_" + k]) < 1e-13, k
                assert _rel(golden["difft_f_" + k], golden["difft_dense_" + k]) < 1e-7, k


def test_loops_reproduce_reference_dispatch(golden, oracle_lib):
    """Kernel.applyK/applyDiffKT of the reference (firstVar = targets) == oracle calls."""
    for tag in golden["kernel_cases"]:
        tag = str(tag)
        name = "gauss" if tag.startswith("gauss") else "laplacian"
        order = int(tag.split("_")[0].replace(name, ""))
        x, y, beta = golden["applyk_x_" + tag], golden["applyk_y_" + tag], golden["applyk_beta_" + tag]
        K = ref.Kernel(name=name, sigma=0.35, order=order)
        np.testing.assert_array_equal(K.applyK(y, beta, firstVar=x), golden["applyk_f_" + tag])
        for na in (1, 3):
            k = "%s_na%d" % (tag, na)
            if "difft_f_" + k in golden.files:
                np.testing.assert_array_equal(K.applyDiffKT(y, golden["difft_a1_" + k], golden["difft_a2_" + k],
                                                            firstVar=x), golden["difft_f_" + k])


def test_dense_weight_loops_match_reference_dense_matrices(golden, oracle_lib):
    """kff.applykmat / applykdiffmat (restated) against the reference's dense
    kernel matrices times the weights, and the reference's dispatch
    (Kernel.applyK(matrixWeights=True), Kernel.applyDiffKmat) == oracle calls."""
    for tag in golden["kernel_cases"]:
        tag = str(tag)
        name = "gauss" if tag.startswith("gauss") else "laplacian"
        order = int(tag.split("_")[0].replace(name, ""))
        x, y = golden["applyk_x_" + tag], golden["applyk_y_" + tag]
        b = golden["kmat_b_" + tag]
        tol = 1e-13 if "laplacian0" not in tag else 2e-9
        oracle_lib.set_exact_coeffs(True)
        try:
            assert _rel(oracle_lib.applykmat(x, y, b, 0.35, order), golden["kmat_dense_" + tag]) < tol, tag
            if "kdiffmat_b_" + tag in golden.files:
                b2 = golden["kdiffmat_b_" + tag]
                assert _rel(oracle_lib.applykdiffmat(x, y, b2, 0.35, order),
                            golden["kdiffmat_dense_" + tag]) < 1e-13, tag
        finally:
            oracle_lib.set_exact_coeffs(False)
        assert _rel(golden["kmat_f_" + tag], golden["kmat_dense_" + tag]) < 5e-8, tag
        K = ref.Kernel(name=name, sigma=0.35, order=order)
        np.testing.assert_array_equal(K.applyK(y, b, firstVar=x, matrixWeights=True), golden["kmat_f_" + tag])
        if "kdiffmat_b_" + tag in golden.files:
            b2 = golden["kdiffmat_b_" + tag]
            assert _rel(golden["kdiffmat_f_" + tag], golden["kdiffmat_dense_" + tag]) < 1e-7, tag
            np.testing.assert_array_equal(K.applyDiffKmat(y, b2, firstVar=x), golden["kdiffmat_f_" + tag])


def test_second_derivative_loops_match_reference(golden, oracle_lib):
    """kff.applykdiff1 / 2 / 1and2 / 11and12 (restated) == the reference's Kernel
    methods on them; the restated applykdiff11 / 12 against the reference's
    independent dense-matrix applyDDiffK11 / 12, and applykdiff1 against the
    dense K' matrix (float32 Fortran literals: ~3e-8 for the Laplacian)."""
    for tag in golden["second_cases"]:
        tag = str(tag)
        name = "gauss" if tag.startswith("gauss") else "laplacian"
        order = int(tag.split("_")[0].replace(name, ""))
        x, a1, a2, p = (golden["sec_%s_%s" % (k, tag)] for k in ("x", "a1", "a2", "p"))
        tol = 1e-13 if name == "gauss" else 1e-7
        np.testing.assert_array_equal(oracle_lib.applykdiff1(x, a1, a2, 0.4, order), golden["sec_kd1_" + tag])
        np.testing.assert_array_equal(oracle_lib.applykdiff2(x, a1, a2, 0.4, order), golden["sec_kd2_" + tag])
        np.testing.assert_array_equal(oracle_lib.applykdiff1and2(x, a1, a2, 0.4, order), golden["sec_kd12_" + tag])
        dx = x[:, None, :] - x[None, :, :]
        r1 = golden["sec_r1_" + tag]
        dense1 = 2 * np.einsum('kl,kl,lj->kj', r1, np.einsum('kld,kd->kl', dx, a1), a2)
        assert _rel(golden["sec_kd1_" + tag], dense1) < tol, tag
        if "sec_dd11_" + tag in golden.files:
            assert _rel(oracle_lib.applykdiff11(x, a1, a2, p, 0.4, order), golden["sec_dd11_" + tag]) < tol, tag
            assert _rel(oracle_lib.applykdiff12(x, a1, a2, p, 0.4, order), golden["sec_dd12_" + tag]) < tol, tag
            np.testing.assert_array_equal(oracle_lib.applykdiff11and12(x, a1, a2, p, 0.4, order),
                                          golden["sec_dd1112_" + tag])


def test_laplacian_order0_derivative_rejected(oracle_lib):
    x = np.zeros((2, 3))
    with pytest.raises(ValueError):
        oracle_lib.applykdifft(x, x, np.ones((1, 2, 3)), np.ones((1, 2, 3)), 1.0, 0)


@pytest.mark.parametrize("kname", ["gauss", "laplacian"])
def test_evolution_matches_reference(golden, oracle_lib, kname):
    p = "evo_%s_" % kname
    K = ref.Kernel(name=kname, sigma=float(golden[p + "sigma"]))
    x0, at, px1 = golden[p + "x0"], golden[p + "at"], golden[p + "px1"]
    np.testing.assert_allclose(ref.landmarkDirectEvolutionEuler(x0, at, K), golden[p + "xt"], rtol=1e-12, atol=1e-13)
    xt2, yt, Jt = ref.landmarkDirectEvolutionEuler(x0, at, K, withJacobian=True, withPointSet=golden[p + "grid"])
    np.testing.assert_allclose(yt, golden[p + "yt"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(Jt, golden[p + "Jt"], rtol=1e-10, atol=1e-12)
    _, nt = ref.landmarkDirectEvolutionEuler(x0, at, K, withNormals=golden[p + "n0"])
    np.testing.assert_allclose(nt, golden[p + "nt"], rtol=1e-12, atol=1e-13)
    _, Jt4 = ref.landmarkDirectEvolutionEuler(x0, at, K, withJacobian=True)
    np.testing.assert_allclose(Jt4, golden[p + "Jt_self"], rtol=1e-10, atol=1e-12)
    pxt, _ = ref.landmarkHamiltonianCovector(x0, at, px1, K, 0.7)
    np.testing.assert_allclose(pxt, golden[p + "pxt"], rtol=1e-12, atol=1e-13)
    dat, _, _ = ref.landmarkHamiltonianGradient(x0, at, px1, K, 0.7, getCovector=True)
    np.testing.assert_allclose(dat, golden[p + "dat"], rtol=1e-12, atol=1e-13)
    xte, ate = ref.landmarkEPDiff(at.shape[0], x0, at[0], K)
    np.testing.assert_allclose(xte, golden[p + "xt_epdiff"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(ate, golden[p + "at_epdiff"], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("kname,sig", [("gauss", 0.4), ("laplacian", 0.5)])
@pytest.mark.parametrize("err", ["current", "measure", "varifold"])
def test_surface_norms_match_reference(golden, oracle_lib, kname, sig, err):
    f = golden["surf_faces"]
    fv1 = ref.Surface(FV=[f, golden["surf_vtgt"]])
    fvD = ref.Surface(FV=[f, golden["surf_vdef"]])
    np.testing.assert_allclose(fvD.centers, golden["surf_centers"], rtol=0, atol=0)
    np.testing.assert_allclose(fvD.surfel, golden["surf_surfel"], rtol=0, atol=0)
    K = ref.Kernel(name=kname, sigma=sig)
    p = "surf_%s_%s_" % (err, kname)
    np.testing.assert_allclose(getattr(ref, err + "Norm0")(fv1, K), golden[p + "norm0"], rtol=1e-12)
    np.testing.assert_allclose(getattr(ref, err + "NormDef")(fvD, fv1, K), golden[p + "normdef"], rtol=1e-12)
    np.testing.assert_allclose(getattr(ref, err + "NormGradient")(fvD, fv1, K), golden[p + "grad"], rtol=1e-11,
                               atol=1e-12)


@pytest.mark.parametrize("kname", ["gauss", "laplacian"])
@pytest.mark.parametrize("err", ["current", "measure"])
def test_curve_norms_match_reference(golden, oracle_lib, kname, err):
    fv1 = ref.Curve(pointSet=golden["curve_vtgt"])
    fvD = ref.Curve(pointSet=golden["curve_vdef"])
    K = ref.Kernel(name=kname, sigma=0.5)
    p = "curve_%s_%s_" % (err, kname)
    np.testing.assert_allclose(getattr(ref, "curve_" + err + "Norm0")(fv1, K), golden[p + "norm0"], rtol=1e-12)
    np.testing.assert_allclose(getattr(ref, "curve_" + err + "NormDef")(fvD, fv1, K), golden[p + "normdef"],
                               rtol=1e-12)
    np.testing.assert_allclose(getattr(ref, "curve_" + err + "NormGradient")(fvD, fv1, K), golden[p + "grad"],
                               rtol=1e-11, atol=1e-12)


@pytest.mark.parametrize("err", ["varifold", "current", "measure"])
def test_surface_matching_trace_matches_reference(golden, oracle_lib, err):
    f, v0, v1 = golden["sm_faces"], golden["sm_v0"], golden["sm_v1"]
    param = ref.MatchingParam(timeStep=0.2, KparDiff=ref.Kernel(name="gauss", sigma=0.4),
                              KparDist=ref.Kernel(name="gauss", sigma=0.3), sigmaError=0.5, errorType=err)
    sm = ref.SurfaceMatching(ref.Surface(FV=[f, v0]), ref.Surface(FV=[f, v1]), param, maxIter=6)
    trace = []
    sm.optimizeMatching(trace=trace)
    p = "sm_%s_" % err
    np.testing.assert_allclose([sm.obj0] + trace, golden[p + "trace"], rtol=1e-9)
    np.testing.assert_allclose(sm.at, golden[p + "at"], rtol=1e-7, atol=1e-10)


@pytest.mark.parametrize("err", ["current", "measure"])
def test_curve_matching_trace_matches_reference(golden, oracle_lib, err):
    param = ref.MatchingParam(timeStep=0.1, KparDiff=ref.Kernel(name="gauss", sigma=0.5),
                              KparDist=ref.Kernel(name="gauss", sigma=0.5), sigmaError=1.0, errorType=err,
                              curves=True)
    cm = ref.CurveMatching(ref.Curve(pointSet=golden["cm_v0"]), ref.Curve(pointSet=golden["cm_v1"]), param,
                           maxIter=8)
    trace = []
    cm.optimizeMatching(trace=trace)
    p = "cm_%s_" % err
    np.testing.assert_allclose([cm.obj0] + trace, golden[p + "trace"], rtol=1e-9)
    np.testing.assert_allclose(cm.at, golden[p + "at"], rtol=1e-7, atol=1e-10)


@pytest.mark.parametrize("err,lam", [("varifold", 1.0), ("current", 0.5)])
def test_template_estimation_trace_matches_reference(golden, oracle_lib, err, lam):
    """surfaceTemplate.py (cg over the prior and three subjects) against the
    reference's own SurfaceTemplate run on the same shapes."""
    f, v0, subs = golden["st_faces"], golden["st_v0"], golden["st_subjects"]
    param = ref.MatchingParam(timeStep=0.2, KparDiff=ref.Kernel(name="gauss", sigma=0.4),
                              KparDist=ref.Kernel(name="gauss", sigma=0.3), sigmaError=0.1, errorType=err)
    st = ref.SurfaceTemplate(ref.Surface(FV=[f, v0]), [ref.Surface(FV=[f, s]) for s in subs], param, maxIter=5,
                             lambdaPrior=lam, testGradient=False)
    trace = []
    st.computeTemplate(trace=trace)
    p = "st_%s_" % err
    assert st.gradEps == golden[p + "gradEps"]
    np.testing.assert_allclose([st.obj0] + trace, golden[p + "trace"], rtol=1e-9)
    np.testing.assert_allclose(st.at, golden[p + "at"], rtol=1e-7, atol=1e-10)
    np.testing.assert_allclose(np.stack(st.atAll), golden[p + "atAll"], rtol=1e-7, atol=1e-10)
    np.testing.assert_allclose(st.fvTmpl.vertices, golden[p + "tmpl"], rtol=1e-9, atol=1e-12)


def test_per_pair_varifold_equals_dense_varifold(oracle_lib):
    """The per-pair varifold functions (for face counts whose F x F arrays do
    not fit) against the dense restatement of surfaces.py:1184-1276."""
    from registration_b200 import geometry as geo
    rng = np.random.default_rng(4)
    v, f = geo.icosphere(2)
    vt = geo.bumped_sphere(v, f, 4, 0.3, 0.1, rng)
    vd = v + 0.03 * rng.standard_normal(v.shape)
    K = ref.Kernel(name="gauss", sigma=0.2)
    a, b = ref.Surface(FV=[f, vd]), ref.Surface(FV=[f, vt])
    n0 = abs(ref.varifoldNorm0(b, K))
    assert abs(ref.varifoldNorm0_pairs(b, K) - ref.varifoldNorm0(b, K)) < 1e-12 * n0
    assert abs(ref.varifoldNormDef_pairs(a, b, K) - ref.varifoldNormDef(a, b, K)) < 1e-12 * n0
    assert _rel(ref.varifoldNormGradient_pairs(a, b, K), ref.varifoldNormGradient(a, b, K)) < 1e-12
