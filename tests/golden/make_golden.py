"""Generates the golden fixtures under tests/golden/ by RUNNING THE REFERENCE.

The reference (saurabh-jain/registration, py-lddmm/) is Python 2 code over an
f2py Fortran module.  In this container there is neither a Python 2
interpreter nor a Fortran compiler, so this script:

1. loads the reference's own Python modules from the read-only reference
   checkout (its py-lddmm/ directory, or $LDDMM_REFERENCE_DIR) after five
   mechanical, semantics-preserving source rewrites done in memory
   (nothing is copied into this repository):
     - tabs expanded to 8-column stops (Python 2 indentation rule);
     - ``print x, y`` statements turned into ``print(x, y)`` calls;
     - ``== None`` / ``!= None`` turned into ``is None`` / ``is not None``
       (what the comparison returned for arrays under the numpy of the
       Python 2 era; modern numpy compares element-wise instead);
     - ``len(x)/2`` turned into ``len(x)//2`` (Python 2 integer division);
     - ``np.mat(`` turned into ``np.asmatrix(`` (the same function under the
       name numpy 2 keeps);
2. registers the oracle (``oracle.FortShim``, a C/OpenMP restatement of
   kernelFunctions.f90) as the module ``kernelFunctions_fort`` that the
   reference imports, and a stub ``gaussianDiffeons`` (imported by
   pointEvolution.py but unused by the landmark functions);
3. runs the reference's Kernel / pointEvolution / surfaces / curves /
   surfaceMatching / curveMatching / conjugateGradient code on small seeded
   inputs, and additionally evaluates the reference's own dense numpy kernel
   matrices (kernelMatrixGauss / kernelMatrixLaplacian) as an independent
   check of the restated Fortran loops.

VTK writers are replaced by no-ops (output only; they do not change the
optimisation state).  Run from the repository root:

    python tests/golden/make_golden.py              # both fixture files
    python tests/golden/make_golden.py --kff-calls  # tests/golden/kff_calls.npz only
    python tests/golden/make_golden.py --extra      # tests/golden/reference_golden_extra.npz only
"""
import io
import os
import re
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from registration_b200 import geometry as geo  # noqa: E402

REF = os.environ.get("LDDMM_REFERENCE_DIR", "/root/reference/py-lddmm")

_PRINT = re.compile(r"^(\s*)print(\s+(.*))?$")


def _py3_source(text):
    out = []
    for line in text.expandtabs(8).splitlines():
        m = _PRINT.match(line)
        if m and not line.strip().startswith("print("):
            body = (m.group(3) or "").rstrip()
            line = "%sprint(%s)" % (m.group(1), body.rstrip(","))
        line = re.sub(r"!=\s*None\b", " is not None", line)
        line = re.sub(r"==\s*None\b", " is None", line)
        line = re.sub(r"(len\([^()]*\))/2\b", r"\1//2", line)
        line = re.sub(r"\bnp\.mat\(", "np.asmatrix(", line)
        out.append(line)
    return "\n".join(out) + "\n"


def load_reference(names=("kernelFunctions", "affineBasis", "pointEvolution", "surfaces", "curves",
                           "matchingParam", "grid", "conjugateGradient", "gradientDescent", "surfaceMatching",
                           "curveMatching", "surfaceTemplate")):
    sys.modules["kernelFunctions_fort"] = oracle.FortShim()
    sys.modules["gaussianDiffeons"] = types.ModuleType("gaussianDiffeons")
    mods = {}
    for nm in names:
        path = os.path.join(REF, nm + ".py")
        with open(path) as fh:
            src = _py3_source(fh.read())
        mod = types.ModuleType(nm)
        mod.__file__ = path
        sys.modules[nm] = mod
        exec(compile(src, path, "exec"), mod.__dict__)
        mods[nm] = mod
    # output-only writers -> no-ops (the VTK writer itself is kept for the mesh cases)
    mods["surfaces_saveVTK2"] = mods["surfaces"].Surface.saveVTK2
    mods["surfaces"].Surface.saveVTK2 = lambda self, *a, **k: None
    mods["curves"].Curve.saveVTK = lambda self, *a, **k: None
    mods["grid"].Grid.saveVTK = lambda self, *a, **k: None
    return mods


def dense_applyk(R, kname, sigma, order, x, y, beta):
    """Reference dense path: kernelMatrix* (kernelFunctions.py:10-198) times beta."""
    kf = R["kernelFunctions"]
    if kname == "gauss":
        K, _ = kf.kernelMatrixGauss(y, firstVar=x, par=[sigma])
    else:
        K, _ = kf.kernelMatrixLaplacian(y, firstVar=x, par=[sigma, order])
    return K @ beta


def dense_applydifft(R, kname, sigma, order, x, y, a1, a2):
    """Reference dense K' matrix (diff=True) with the formula kept beside the
    f2py call at kernelFunctions.py:424-430."""
    kf = R["kernelFunctions"]
    if kname == "gauss":
        r, _ = kf.kernelMatrixGauss(y, firstVar=x, par=[sigma], diff=True)
    else:
        r, _ = kf.kernelMatrixLaplacian(y, firstVar=x, par=[sigma, order], diff=True)
    a = sum(a1[i] @ a2[i].T for i in range(a1.shape[0]))
    g1 = r * a
    return 2 * (x * g1.sum(axis=1)[:, None] - g1 @ y)


def dense_kmat(R, kname, sigma, order, x, y, diff=False):
    """The reference's dense kernel matrix (or K' matrix with diff=True)."""
    kf = R["kernelFunctions"]
    if kname == "gauss":
        K, _ = kf.kernelMatrixGauss(y, firstVar=x, par=[sigma], diff=diff)
    else:
        K, _ = kf.kernelMatrixLaplacian(y, firstVar=x, par=[sigma, order], diff=diff)
    return K


def kernel_cases(R, out):
    kf = R["kernelFunctions"]
    rng = np.random.default_rng(1234)
    rng_mat = np.random.default_rng(4321)   # dense-weight cases (separate stream)
    cases = []
    for kname, order in [("gauss", 10), ("laplacian", 0), ("laplacian", 1), ("laplacian", 2), ("laplacian", 3),
                         ("laplacian", 4)]:
        for d in (2, 3):
            for dimb in (1, 3):
                n, m = 37, 53
                sigma = 0.35
                x = rng.uniform(0, 1, (n, d))
                y = rng.uniform(0, 1, (m, d))
                y[:5] = x[:5]          # exact coincidences: zero-distance branch
                y[5] = x[6] + 1e-10    # below the 1e-8 threshold
                beta = rng.standard_normal((m, dimb))
                K = kf.Kernel(name=kname, sigma=sigma, order=order)
                fk = K.applyK(y, beta, firstVar=x)
                fself = K.applyK(x, rng.standard_normal((n, dimb)))
                tag = "%s%d_d%d_b%d" % (kname, K.order, d, dimb)
                out["applyk_x_" + tag] = x
                out["applyk_y_" + tag] = y
                out["applyk_beta_" + tag] = beta
                out["applyk_f_" + tag] = fk
                oracle.set_exact_coeffs(True)
                out["applyk_dense_" + tag] = dense_applyk(R, kname, sigma, K.order, x, y, beta)
                out["applyk_exact_" + tag] = oracle.applyk(x, y, beta, sigma, K.order)
                oracle.set_exact_coeffs(False)
                # dense weights: Kernel.applyK(matrixWeights=True) -> kff.applykmat
                bmat = rng_mat.standard_normal((n, m, dimb))
                out["kmat_b_" + tag] = bmat
                out["kmat_f_" + tag] = K.applyK(y, bmat, firstVar=x, matrixWeights=True)
                Kd = dense_kmat(R, kname, sigma, K.order, x, y)
                out["kmat_dense_" + tag] = (Kd[:, :, None] * bmat).sum(axis=1)
                if K.order > 0 and dimb == 1:
                    # Kernel.applyDiffKmat -> kff.applykdiffmat
                    b2 = rng_mat.standard_normal((n, m))
                    out["kdiffmat_b_" + tag] = b2
                    out["kdiffmat_f_" + tag] = K.applyDiffKmat(y, b2, firstVar=x)
                    g = dense_kmat(R, kname, sigma, K.order, x, y, diff=True) * b2
                    out["kdiffmat_dense_" + tag] = 2 * (x * g.sum(axis=1)[:, None] - g @ y)
                if K.order > 0:
                    for na in (1, 3):
                        a1 = rng.standard_normal((na, n, dimb))
                        a2 = rng.standard_normal((na, m, dimb))
                        fd = K.applyDiffKT(y, a1, a2, firstVar=x)
                        t2 = tag + "_na%d" % na
                        out["difft_a1_" + t2] = a1
                        out["difft_a2_" + t2] = a2
                        out["difft_f_" + t2] = fd
                        oracle.set_exact_coeffs(True)
                        out["difft_dense_" + t2] = dense_applydifft(R, kname, sigma, K.order, x, y, a1, a2)
                        out["difft_exact_" + t2] = oracle.applykdifft(x, y, a1, a2, sigma, K.order)
                        oracle.set_exact_coeffs(False)
                cases.append(tag)
                del fself
    out["kernel_cases"] = np.array(cases)


def second_cases(R, out):
    """First / second derivative loops (kff.applykdiff1, 2, 1and2, 11and12 through
    the reference's Kernel methods) and the reference's dense-matrix
    applyDDiffK11 / applyDDiffK12 (kernelFunctions.py:459-507)."""
    kf = R["kernelFunctions"]
    rng = np.random.default_rng(777)
    cases = []
    for kname, order in [("gauss", 10), ("laplacian", 1), ("laplacian", 2), ("laplacian", 3), ("laplacian", 4)]:
        for d in (2, 3):
            n = 41
            x = rng.uniform(0, 1, (n, d))
            x[4] = x[3]                       # coincident points: zero-distance branch
            a1, a2, p = (rng.standard_normal((n, d)) for _ in range(3))
            K = kf.Kernel(name=kname, sigma=0.4, order=order)
            tag = "%s%d_d%d" % (kname, K.order, d)
            out["sec_x_" + tag], out["sec_a1_" + tag], out["sec_a2_" + tag], out["sec_p_" + tag] = x, a1, a2, p
            out["sec_kd1_" + tag] = K.applyDiffK(x, a1, a2)
            out["sec_kd2_" + tag] = K.applyDiffK2(x, a1, a2)
            out["sec_kd12_" + tag] = K.applyDiffK1and2(x, a1, a2)
            out["sec_r1_" + tag] = dense_kmat(R, kname, 0.4, K.order, x, x, diff=True)
            if K.order >= 2:
                out["sec_dd1112_" + tag] = K.applyDDiffK11and12(x, a1, a2, p)
                out["sec_dd11_" + tag] = K.applyDDiffK11(x, a1, a2, p)
                out["sec_dd12_" + tag] = K.applyDDiffK12(x, a1, a2, p)
            cases.append(tag)
    out["second_cases"] = np.array(cases)


def second_order_cases(R, out):
    """secondOrderEvolution / Hamiltonian / Covector / Gradient (pointEvolution.py:882-1091),
    one target time (nTarg = 1) and a `times` argument (the reference's
    times=None branch raises on `range(nTarg) + 1`)."""
    ev = R["pointEvolution"]
    kf = R["kernelFunctions"]
    rng = np.random.default_rng(2468)
    for kname, order in [("gauss", 10), ("laplacian", 3)]:
        n, d, T = 30, 3, 5
        x0 = rng.uniform(0, 1, (n, d))
        a0 = 0.3 * rng.standard_normal((n, d))
        rhot = 0.2 * rng.standard_normal((T, n, d))
        px1 = [rng.standard_normal((n, d))]
        pa1 = [rng.standard_normal((n, d))]
        K = kf.Kernel(name=kname, sigma=0.5, order=order)
        pre = "so_%s_" % kname
        out[pre + "x0"], out[pre + "a0"], out[pre + "rhot"] = x0, a0, rhot
        out[pre + "px1"], out[pre + "pa1"] = px1[0], pa1[0]
        xt, at = ev.secondOrderEvolution(x0, a0, rhot, K)
        out[pre + "xt"], out[pre + "at"] = xt, at
        out[pre + "H"] = np.array(ev.secondOrderHamiltonian(xt[2], at[2], rhot[2], px1[0], pa1[0], K))
        pxt, pat, _, _ = ev.secondOrderCovector(x0, a0, rhot, px1, pa1, K, times=np.ones(1))
        out[pre + "pxt"], out[pre + "pat"] = pxt, pat
        da0, drhot, _, _ = ev.secondOrderGradient(x0, a0, rhot, px1, pa1, K, times=np.ones(1))
        out[pre + "da0"], out[pre + "drhot"] = da0, drhot


def evolution_cases(R, out):
    kf = R["kernelFunctions"]
    ev = R["pointEvolution"]
    rng = np.random.default_rng(99)
    for kname, sigma in [("gauss", 0.5), ("laplacian", 0.6)]:
        N, d, T = 40, 3, 5
        x0 = rng.uniform(-1, 1, (N, d))
        at = 0.3 * rng.standard_normal((T, N, d))
        px1 = rng.standard_normal((N, d))
        K = kf.Kernel(name=kname, sigma=sigma)
        xt = ev.landmarkDirectEvolutionEuler(x0, at, K)
        grid = rng.uniform(-1, 1, (17, d))
        xt2, yt, Jt = ev.landmarkDirectEvolutionEuler(x0, at, K, withJacobian=True, withPointSet=grid)
        n0 = rng.standard_normal((N, d))
        xt3, nt = ev.landmarkDirectEvolutionEuler(x0, at, K, withNormals=n0)
        xt4, Jt4 = ev.landmarkDirectEvolutionEuler(x0, at, K, withJacobian=True)
        pxt, xt5 = ev.landmarkHamiltonianCovector(x0, at, px1, K, 0.7)
        dat, xt6, pxt6 = ev.landmarkHamiltonianGradient(x0, at, px1, K, 0.7, getCovector=True)
        xte, ate = ev.landmarkEPDiff(T, x0, at[0], K)
        p = "evo_%s_" % kname
        for k, v in dict(x0=x0, at=at, px1=px1, xt=xt, grid=grid, yt=yt, Jt=Jt, n0=n0, nt=nt, Jt_self=Jt4,
                         pxt=pxt, dat=dat, xt_epdiff=xte, at_epdiff=ate).items():
            out[p + k] = v
        out[p + "sigma"] = sigma


def surface_cases(R, out):
    kf = R["kernelFunctions"]
    sf = R["surfaces"]
    rng = np.random.default_rng(7)
    v, f = geo.icosphere(1)
    vt = geo.bumped_sphere(v, f, 4, 0.5, 0.2, rng)
    vd = v + 0.05 * rng.standard_normal(v.shape)
    fv1 = sf.Surface(FV=[f, vt])
    fvD = sf.Surface(FV=[f, vd])
    out["surf_faces"] = f
    out["surf_vdef"] = vd
    out["surf_vtgt"] = vt
    out["surf_centers"] = fvD.centers
    out["surf_surfel"] = fvD.surfel
    for kname, sig in [("gauss", 0.4), ("laplacian", 0.5)]:
        K = kf.Kernel(name=kname, sigma=sig)
        for err in ("current", "measure", "varifold"):
            p = "surf_%s_%s_" % (err, kname)
            out[p + "norm0"] = getattr(sf, err + "Norm0")(fv1, K)
            out[p + "normdef"] = getattr(sf, err + "NormDef")(fvD, fv1, K)
            out[p + "grad"] = getattr(sf, err + "NormGradient")(fvD, fv1, K)


def curve_cases(R, out):
    kf = R["kernelFunctions"]
    cv = R["curves"]
    rng = np.random.default_rng(11)
    v, f = geo.ellipse_curve(48)
    vt, _ = geo.bumped_curve(v, 4, 0.3, 0.1, rng)
    vd = v + 0.03 * rng.standard_normal(v.shape)
    fv1 = cv.Curve(pointSet=vt)
    fvD = cv.Curve(pointSet=vd)
    out["curve_vdef"] = vd
    out["curve_vtgt"] = vt
    for kname, sig in [("gauss", 0.5), ("laplacian", 0.5)]:
        K = kf.Kernel(name=kname, sigma=sig)
        for err in ("current", "measure"):
            p = "curve_%s_%s_" % (err, kname)
            out[p + "norm0"] = getattr(cv, err + "Norm0")(fv1, K)
            out[p + "normdef"] = getattr(cv, err + "NormDef")(fvD, fv1, K)
            out[p + "grad"] = getattr(cv, err + "NormGradient")(fvD, fv1, K)


def _record_trace(obj):
    trace = []
    orig = obj.acceptVarTry

    def accept():
        orig()
        trace.append(float(obj.obj))

    obj.acceptVarTry = accept
    return trace


def matching_cases(R, out):
    kf = R["kernelFunctions"]
    sf = R["surfaces"]
    cv = R["curves"]
    SM = R["surfaceMatching"]
    CM = R["curveMatching"]
    tmp = tempfile.mkdtemp(prefix="lddmm_golden_")
    # surface matching, icosphere subdivision 2 (162 vertices)
    rng = np.random.default_rng(5)
    v, f = geo.icosphere(2)
    vt = geo.bumped_sphere(v, f, 6, 0.35, 0.15, rng)
    out["sm_faces"] = f
    out["sm_v0"] = v
    out["sm_v1"] = vt
    for err, sdist in [("varifold", 0.3), ("current", 0.3), ("measure", 0.3)]:
        param = SM.SurfaceMatchingParam(timeStep=0.2, KparDiff=kf.Kernel(name="gauss", sigma=0.4),
                                        KparDist=kf.Kernel(name="gauss", sigma=sdist), sigmaError=0.5,
                                        errorType=err)
        sm = SM.SurfaceMatching(Template=sf.Surface(FV=[f, v]), Target=sf.Surface(FV=[f, vt]), param=param,
                                maxIter=6, testGradient=False, outputDir=tmp)
        sm.saveRate = 10 ** 9   # skip the output-only branch of endOfIteration
        trace = _record_trace(sm)
        sm.optimizeMatching()
        p = "sm_%s_" % err
        out[p + "trace"] = np.array([float(sm.obj0)] + trace)
        out[p + "at"] = sm.at
        out[p + "gradEps"] = sm.gradEps
    # curve matching, 64-vertex ellipse (curveMatching.py: cg with epsInit=10)
    rng = np.random.default_rng(3)
    v, f = geo.ellipse_curve(64)
    vt, _ = geo.bumped_curve(v, 4, 0.3, 0.1, rng)
    out["cm_v0"] = v
    out["cm_v1"] = vt
    for err in ("current", "measure"):
        param = CM.CurveMatchingParam(timeStep=0.1, KparDiff=kf.Kernel(name="gauss", sigma=0.5),
                                      KparDist=kf.Kernel(name="gauss", sigma=0.5), sigmaError=1.0, errorType=err)
        stdout = sys.stdout
        sys.stdout = io.StringIO()   # the reference prints on every objectiveFun
        try:
            cm = CM.CurveMatching(Template=cv.Curve(pointSet=v), Target=cv.Curve(pointSet=vt), param=param,
                                  maxIter=8, saveRate=0, outputDir=tmp)
            trace = _record_trace(cm)
            cm.optimizeMatching()
        finally:
            sys.stdout = stdout
        p = "cm_%s_" % err
        out[p + "trace"] = np.array([float(cm.obj0)] + trace)
        out[p + "at"] = cm.at
        out[p + "gradEps"] = cm.gradEps


def template_cases(R, out):
    """Template estimation (surfaceTemplate.py) on three bumped icospheres.  The
    reference's SurfaceTemplate never sets two attributes that the inherited
    SurfaceMatching.objectiveFunDef reads (x0, used by the prior's shot, and
    the velocity store v); they are set on the instance to the hyper-template's
    vertices and a zero store before the run."""
    kf = R["kernelFunctions"]
    sf = R["surfaces"]
    SM = R["surfaceMatching"]
    ST = R["surfaceTemplate"]
    tmp = tempfile.mkdtemp(prefix="lddmm_golden_")
    rng = np.random.default_rng(11)
    v, f = geo.icosphere(2)
    subjects = [geo.bumped_sphere(v, f, 5, 0.4, 0.2, rng) for _ in range(3)]
    out["st_faces"] = f
    out["st_v0"] = v
    out["st_subjects"] = np.stack(subjects)
    for err, lam in [("varifold", 1.0), ("current", 0.5)]:
        param = SM.SurfaceMatchingParam(timeStep=0.2, KparDiff=kf.Kernel(name="gauss", sigma=0.4),
                                        KparDist=kf.Kernel(name="gauss", sigma=0.3), sigmaError=0.1,
                                        errorType=err)
        st = ST.SurfaceTemplate(HyperTmpl=sf.Surface(FV=[f, v]), Targets=[sf.Surface(FV=[f, s]) for s in subjects],
                                param=param, maxIter=5, lambdaPrior=lam, verb=False, outputDir=tmp)
        st.x0 = np.copy(st.fv0.vertices)
        st.v = np.zeros((st.Tsize, st.npt, st.dim))
        trace = _record_trace(st)
        np.random.seed(7)      # cg's TestGradient direction (logged only)
        st.computeTemplate()
        p = "st_%s_" % err
        out[p + "trace"] = np.array([float(st.obj0)] + trace)
        out[p + "at"] = np.copy(st.at)
        out[p + "atAll"] = np.stack(st.atAll)
        out[p + "gradEps"] = st.gradEps
        out[p + "tmpl"] = np.copy(st.fvTmpl.vertices)


def mesh_cases(R, out):
    """Mesh files and per-vertex geometry (surfaces.py:77-139, 711-925) on a
    perturbed, decimated icosphere (obtuse faces, odd vertex count).  The
    reference's readbyu calls scipy.fabs, one of the numpy functions that
    scipy re-exported in the Python 2 era; numpy's fabs is bound in its
    place for the run."""
    sf = R["surfaces"]
    sf.sp = types.SimpleNamespace(fabs=np.fabs)
    tmp = tempfile.mkdtemp(prefix="lddmm_golden_")
    rng = np.random.default_rng(21)
    v, f = geo.icosphere(3)
    v, f = geo.decimate(v + 0.02 * rng.standard_normal(v.shape), f, 301, rng)
    out["mesh_v"] = v
    out["mesh_f"] = f
    fv = sf.Surface(FV=[f, v])
    AV, AF = fv.computeVertexArea()
    out["mesh_AV"] = AV
    out["mesh_AF"] = AF
    out["mesh_normals"] = fv.computeVertexNormals()
    out["mesh_volume"] = fv.surfVolume()
    byu = os.path.join(tmp, "m.byu")
    fv.savebyu(byu)
    with open(byu) as fh:
        out["mesh_byu_text"] = np.array(fh.read())
    back = sf.Surface(filename=byu)
    out["mesh_byu_v"] = back.vertices
    out["mesh_byu_f"] = back.faces
    vtk = os.path.join(tmp, "m.vtk")
    sf.Surface.saveVTK2 = R["surfaces_saveVTK2"]
    fv.saveVTK(vtk, scalars=AV[:, 0], normals=out["mesh_normals"], vectors=0.5 * out["mesh_normals"])
    sf.Surface.saveVTK2 = lambda self, *a, **k: None
    with open(vtk) as fh:
        out["mesh_vtk_text"] = np.array(fh.read())
    off_lines = ["# written for the golden fixtures", "OFF", "# counts", "%d %d 0" % (len(v), len(f))]
    off_lines += ["%.17g %.17g %.17g" % tuple(p) for p in v]
    off_lines += ["# faces"] + ["3 %d %d %d" % tuple(t) for t in f]
    off = os.path.join(tmp, "m.off")
    with open(off, "w") as fh:
        fh.write("\n".join(off_lines) + "\n")
    out["mesh_off_text"] = np.array("\n".join(off_lines) + "\n")
    back = sf.Surface(filename=off)
    out["mesh_off_v"] = back.vertices
    out["mesh_off_f"] = back.faces


class _KffRecorder:
    """Stands in for the module ``kernelFunctions_fort`` of the reference's
    kernelFunctions.py and records every call it receives (routine name, the
    positional arguments exactly as the reference passes them, the result of
    the oracle), at most `cap` calls per routine."""

    def __init__(self, inner, cap=12):
        self.inner, self.cap, self.calls, self.count = inner, cap, [], {}

    def __getattr__(self, name):
        fn = getattr(self.inner, name)

        def call(*args):
            res = fn(*args)
            if self.count.get(name, 0) < self.cap:
                self.count[name] = self.count.get(name, 0) + 1
                self.calls.append((name, [np.array(a, copy=True) for a in args], np.array(res, copy=True)))
            return res
        return call


def kff_call_cases(R):
    """The calls the reference's own Python makes into kernelFunctions_fort
    (Kernel.applyK / applyDiffKT / applyDiffKmat / applyDiffK*, through
    landmarkHamiltonianGradient, the surface varifold and current gradients and
    the curve current gradient), with the oracle's results, for replaying them
    through a drop-in module."""
    kf = R["kernelFunctions"]
    ev = R["pointEvolution"]
    sf = R["surfaces"]
    cv = R["curves"]
    rec = _KffRecorder(oracle.FortShim())
    saved = kf.kff
    kf.kff = rec
    try:
        rng = np.random.default_rng(99)
        x, y = rng.uniform(0, 1, (40, 3)), rng.uniform(0, 1, (55, 3))
        for K in (kf.Kernel(name="gauss", sigma=0.3), kf.Kernel(name="laplacian", sigma=0.3, order=2)):
            K.applyK(y, rng.standard_normal((55, 3)))
            K.applyK(y, rng.standard_normal((55, 1)), firstVar=x)
            K.applyDiffKT(y, rng.standard_normal((1, 40, 3)), rng.standard_normal((1, 55, 3)), firstVar=x)
            K.applyDiffK(x, rng.standard_normal((40, 3)), rng.standard_normal((40, 3)))
            K.applyDiffK2(x, rng.standard_normal((40, 3)), rng.standard_normal((40, 3)))
            K.applyDiffK1and2(x, rng.standard_normal((40, 3)), rng.standard_normal((40, 3)))
            K.applyDDiffK11and12(x, rng.standard_normal((40, 3)), rng.standard_normal((40, 3)),
                                 rng.standard_normal((40, 3)))
        K = kf.Kernel(name="gauss", sigma=0.5)
        x0 = rng.uniform(-1, 1, (30, 3))
        ev.landmarkHamiltonianGradient(x0, 0.2 * rng.standard_normal((3, 30, 3)), rng.standard_normal((30, 3)), K,
                                       1.0)
        v, f = geo.icosphere(1)
        vt = geo.bumped_sphere(v, f, 3, 0.4, 0.1, rng)
        a, b = sf.Surface(FV=[f, v + 0.02 * rng.standard_normal(v.shape)]), sf.Surface(FV=[f, vt])
        KD = kf.Kernel(name="gauss", sigma=0.4)
        sf.varifoldNormGradient(a, b, KD)
        sf.currentNormGradient(a, b, KD)
        c, _ = geo.ellipse_curve(24)
        ct, _ = geo.bumped_curve(c, 2, 0.3, 0.1, rng)
        cv.currentNormGradient(cv.Curve(pointSet=c), cv.Curve(pointSet=ct), kf.Kernel(name="laplacian", sigma=0.5,
                                                                                       order=3))
    finally:
        kf.kff = saved
    out = {"ncalls": np.array(len(rec.calls))}
    for i, (name, args, res) in enumerate(rec.calls):
        out["c%d_name" % i] = np.array(name)
        out["c%d_nargs" % i] = np.array(len(args))
        for j, a in enumerate(args):
            out["c%d_a%d" % (i, j)] = a
        out["c%d_out" % i] = res
    return out


def extra_cases(R):
    """Reference outputs of the options that the main fixtures do not cover:
    landmarkEPDiff with a point set, normals and the Jacobian
    (pointEvolution.py:599-658), and the affine / euclidean parts of
    Kernel.applyK and the euclidean part of Kernel.applyDiffKT
    (kernelFunctions.py:334-367, 431-448)."""
    kf = R["kernelFunctions"]
    ev = R["pointEvolution"]
    out = {}
    rng = np.random.default_rng(77)
    for kname, sigma in [("gauss", 0.5), ("laplacian", 0.6)]:
        N, d, T = 40, 3, 6
        x0 = rng.uniform(-1, 1, (N, d))
        a0 = 0.3 * rng.standard_normal((N, d))
        grid = rng.uniform(-1, 1, (17, d))
        n0 = rng.standard_normal((N, d))
        K = kf.Kernel(name=kname, sigma=sigma)
        xt, at, yt, nt, Jt = ev.landmarkEPDiff(T, x0, a0, K, withJacobian=True, withNormals=n0, withPointSet=grid)
        xt2, at2, Jt2 = ev.landmarkEPDiff(T, x0, a0, K, withJacobian=True)
        p = "epd_%s_" % kname
        for k, v in dict(x0=x0, a0=a0, grid=grid, n0=n0, xt=xt, at=at, yt=yt, nt=nt, Jt=Jt, Jt_only=Jt2).items():
            out[p + k] = v
        out[p + "sigma"] = sigma
    cases = []
    for affine in ("affine", "euclidean"):
        for d in (2, 3):
            for kname in ("gauss", "laplacian"):
                tag = "%s_%s_d%d" % (affine, kname, d)
                n, m = 23, 31
                x = rng.uniform(-1, 1, (m, d))    # sources
                y = rng.uniform(-1, 1, (n, d))    # targets
                a = rng.standard_normal((m, d))
                K = kf.Kernel(name=kname, sigma=0.4, affine=affine, w1=0.7, w2=1.3, dim=d,
                              center=list(rng.uniform(-0.2, 0.2, d)))
                out["aff_x_" + tag], out["aff_y_" + tag], out["aff_a_" + tag] = x, y, a
                out["aff_center_" + tag] = np.asarray(K.center, dtype=np.float64)
                try:
                    out["aff_k_" + tag] = K.applyK(x, a)
                except ValueError:
                    # euclidean, firstVar None: the reference multiplies np.matrix objects
                    # ((xE * a).sum() is a matrix product, kernelFunctions.py:360) and fails
                    pass
                out["aff_kf_" + tag] = K.applyK(x, a, firstVar=y)
                if affine == "euclidean":
                    a1 = rng.standard_normal((2, n, d))
                    a2 = rng.standard_normal((2, m, d))
                    out["aff_a1_" + tag], out["aff_a2_" + tag] = a1, a2
                    out["aff_dkt_" + tag] = K.applyDiffKT(x, a1, a2, firstVar=y)
                    b1 = rng.standard_normal((1, m, d))
                    b2 = rng.standard_normal((1, m, d))
                    out["aff_b1_" + tag], out["aff_b2_" + tag] = b1, b2
                    out["aff_dkts_" + tag] = K.applyDiffKT(x, b1, b2)
                cases.append(tag)
    out["aff_cases"] = np.array(cases)
    return out


def write_extra(R):
    extra = extra_cases(R)
    dst = os.path.join(HERE, "reference_golden_extra.npz")
    np.savez_compressed(dst, **extra)
    print("wrote %s (%d arrays, %.1f KB)" % (dst, len(extra), os.path.getsize(dst) / 1024.0))


def write_kff_calls(R):
    calls = kff_call_cases(R)
    dst = os.path.join(HERE, "kff_calls.npz")
    np.savez_compressed(dst, **calls)
    print("wrote %s (%d calls, %.1f KB)" % (dst, int(calls["ncalls"]), os.path.getsize(dst) / 1024.0))


def main():
    oracle.build()
    oracle.set_num_threads(4)
    R = load_reference()
    if "--kff-calls" in sys.argv:     # only the recorded kernelFunctions_fort calls
        write_kff_calls(R)
        return
    if "--extra" in sys.argv:         # only tests/golden/reference_golden_extra.npz
        write_extra(R)
        return
    out = {}
    kernel_cases(R, out)
    second_cases(R, out)
    second_order_cases(R, out)
    evolution_cases(R, out)
    surface_cases(R, out)
    curve_cases(R, out)
    matching_cases(R, out)
    template_cases(R, out)
    mesh_cases(R, out)
    dst = os.path.join(HERE, "reference_golden.npz")
    np.savez_compressed(dst, **out)
    print("wrote %s (%d arrays, %.1f KB)" % (dst, len(out), os.path.getsize(dst) / 1024.0))
    write_kff_calls(R)
    write_extra(R)


if __name__ == "__main__":
    main()
