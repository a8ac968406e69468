"""Oracle numpy transliteration -- TEST INFRASTRUCTURE ONLY.

Python-3 / numpy restatement, in FP64, of the py-lddmm layers that sit above
the Fortran loops on the point-LDDMM hot path.  Each function cites the
reference lines it follows (paths relative to the reference project).  The
pairwise sums go through the C oracle (``oracle.applyk`` ...), exactly as the
reference goes through ``kernelFunctions_fort``.

Only the ``affine='none'`` configuration is restated (the one every benchmark
configuration uses); file output (VTK writers in endOfIteration) is left out
because it does not change the optimisation state.
"""
import logging

import numpy as np

import oracle as _o


# ---------------------------------------------------------------------------
# Kernel (py-lddmm/kernelFunctions.py:238-530)
# ---------------------------------------------------------------------------
class Kernel:
    """KernelSpec/Kernel (kernelFunctions.py:238-307): Gaussian forces
    order 10 (:263), Laplacian orders above 4 fall back to 3 (:258-259)."""

    def __init__(self, name='gauss', affine='none', sigma=6.5, order=10, w1=1.0, w2=1.0, dim=3, center=(0, 0, 0),
                 weight=1.0):
        self.name = name
        self.sigma = sigma
        self.order = order
        self.weight = weight
        self.affine = affine
        if affine != 'none':
            raise NotImplementedError("oracle restates affine='none' only")
        if name == 'laplacian':
            if self.order > 4:
                self.order = 3
        elif name == 'gauss':
            self.order = 10
        else:
            self.name = 'none'

    # kernelFunctions.py:310-369
    def applyK(self, x, a, firstVar=None, grid=None, matrixWeights=False):
        if self.name == 'none':
            return np.zeros([x.shape[0], a.shape[1]])
        tgt = x if firstVar is None else firstVar
        if matrixWeights:
            return _o.applykmat(tgt, x, a, self.sigma, self.order)
        return _o.applyk(tgt, x, a, self.sigma, self.order)

    # kernelFunctions.py:405-410
    def applyDiffKmat(self, x, beta, firstVar=None):
        tgt = x if firstVar is None else firstVar
        return _o.applykdiffmat(tgt, x, beta, self.sigma, self.order)

    # kernelFunctions.py:413-449 (affine 'none')
    def applyDiffKT(self, x, a1, a2, firstVar=None):
        a1 = np.asarray(a1)
        a2 = np.asarray(a2)
        tgt = x if firstVar is None else firstVar
        return _o.applykdifft(tgt, x, a1, a2, self.sigma, self.order)

    # kernelFunctions.py:391-402, 452-454
    def applyDiffK(self, x, a1, a2):
        return _o.applykdiff1(x, a1, a2, self.sigma, self.order)

    def applyDiffK2(self, x, a1, a2):
        return _o.applykdiff2(x, a1, a2, self.sigma, self.order)

    def applyDiffK1and2(self, x, a1, a2):
        return _o.applykdiff1and2(x, a1, a2, self.sigma, self.order)

    def applyDDiffK11and12(self, x, n, a, p):
        return _o.applykdiff11and12(x, n, a, p, self.sigma, self.order)

    # kernelFunctions.py:510-530: dense K' matrix (precompute(diff=True) * weight)
    def applyDivergence(self, x, a, firstVar=None):
        tgt = x if firstVar is None else firstVar
        r = kernel_matrix_diff(self, tgt, x) * self.weight
        ra = r @ a
        return 2 * ((ra * tgt).sum(axis=1) - r @ (a * x).sum(axis=1))


def kernel_matrix(K, x, y):
    """Dense K(x_k, y_l), exact-rational Laplacian polynomials
    (kernelMatrixGauss / kernelMatrixLaplacian, kernelFunctions.py:10-198)."""
    d2 = ((x[:, None, :] - y[None, :, :]) ** 2).sum(axis=2)
    if K.name == 'gauss':
        return np.exp(-d2 / (2 * K.sigma ** 2))
    u = np.sqrt(d2) / K.sigma
    pol = {0: lambda u: 1.0 + 0 * u, 1: lambda u: 1. + u, 2: lambda u: (3. + 3 * u + u * u) / 3.,
           3: lambda u: (15. + 15 * u + 6 * u * u + u * u * u) / 15.,
           4: lambda u: (105. + 105 * u + 45 * u * u + 10 * u ** 3 + u ** 4) / 105.}[K.order]
    return pol(u) * np.exp(-u)


def kernel_matrix_diff(K, x, y):
    """Dense K'(x_k, y_l) (kernelFunctions.py:10-55, 75-88, 152-185 with diff=True)."""
    d2 = ((x[:, None, :] - y[None, :, :]) ** 2).sum(axis=2)
    s2 = 2 * K.sigma ** 2
    if K.name == 'gauss':
        return -np.exp(-d2 / s2) / s2
    u = np.sqrt(d2) / K.sigma
    pol = {1: lambda u: 1. + 0 * u, 2: lambda u: (1 + u) / 3., 3: lambda u: (3 + 3 * u + u * u) / 15.,
           4: lambda u: (15 + 15 * u + 6 * u * u + u ** 3) / 105.}[K.order]
    return -pol(u) * np.exp(-u) / s2


# ---------------------------------------------------------------------------
# Point evolution (py-lddmm/pointEvolution.py)
# ---------------------------------------------------------------------------
def landmarkDirectEvolutionEuler(x0, at, KparDiff, affine=None, withJacobian=False, withNormals=None,
                                 withPointSet=None):
    """pointEvolution.py:666-730: x_{k+1} = x_k + dt K(x_k,x_k) a_k, dt = 1/T."""
    N = x0.shape[0]
    dim = x0.shape[-1]
    M = at.shape[0] + 1
    timeStep = 1.0 / (M - 1)
    xt = np.zeros([M, N, dim])
    xt[0] = x0
    simple = True
    if withNormals is not None:
        simple = False
        nt = np.zeros([M, N, dim])
        nt[0] = withNormals
    if withPointSet is not None:
        simple = False
        K = withPointSet.shape[0]
        yt = np.zeros([M, K, dim])
        yt[0] = withPointSet
        if withJacobian:
            Jt = np.zeros([M, K])
    elif withJacobian:
        simple = False
        Jt = np.zeros([M, N])
    for k in range(M - 1):
        z = xt[k]
        a = at[k]
        xt[k + 1] = z + timeStep * KparDiff.applyK(z, a)
        if affine is not None:
            xt[k + 1] += timeStep * (z @ affine[0][k].T + affine[1][k])
        if withPointSet is not None:
            zy = yt[k]
            yt[k + 1] = zy + timeStep * KparDiff.applyK(z, a, firstVar=zy)
            if affine is not None:
                yt[k + 1] += timeStep * (zy @ affine[0][k].T + affine[1][k])
            if withJacobian:
                Jt[k + 1] = Jt[k] + timeStep * KparDiff.applyDivergence(z, a, firstVar=zy)
        elif withJacobian:
            Jt[k + 1] = Jt[k] + timeStep * KparDiff.applyDivergence(z, a)
        if withNormals is not None:
            zn = nt[k]
            nt[k + 1] = zn - timeStep * KparDiff.applyDiffKT(z, zn[np.newaxis], a[np.newaxis])
            if affine is not None:
                nt[k + 1] += timeStep * (zn @ affine[0][k])
    if simple:
        return xt
    out = [xt]
    if withPointSet is not None:
        out.append(yt)
    if withNormals is not None:
        out.append(nt)
    if withJacobian:
        out.append(Jt)
    return out


def landmarkEPDiff(T, x0, a0, KparDiff):
    """pointEvolution.py:599-658 (no affine / extra outputs)."""
    N, dim = x0.shape
    timeStep = 1.0 / T
    at = np.zeros([T, N, dim])
    xt = np.zeros([T + 1, N, dim])
    xt[0] = x0
    at[0] = a0
    for k in range(T):
        z = xt[k]
        a = at[k]
        xt[k + 1] = z + timeStep * KparDiff.applyK(z, a)
        if k < T - 1:
            at[k + 1] = a - timeStep * KparDiff.applyDiffKT(z, a[np.newaxis], a[np.newaxis])
    return xt, at


def landmarkHamiltonianCovector(x0, at, px1, KparDiff, regweight, affine=None):
    """pointEvolution.py:735-765: backward sweep
    p_t = p_{t+1} + dt applyDiffKT(x_t, [p, a, -2 rw a], [a, p, a])."""
    N, dim = x0.shape
    M = at.shape[0]
    timeStep = 1.0 / M
    xt = landmarkDirectEvolutionEuler(x0, at, KparDiff, affine=affine)
    pxt = np.zeros([M + 1, N, dim])
    pxt[M] = px1
    for t in range(M):
        px = pxt[M - t]
        z = xt[M - t - 1]
        a = at[M - t - 1]
        a1 = np.concatenate((px[np.newaxis], a[np.newaxis], -2 * regweight * a[np.newaxis]))
        a2 = np.concatenate((a[np.newaxis], px[np.newaxis], a[np.newaxis]))
        zpx = KparDiff.applyDiffKT(z, a1, a2)
        pxt[M - t - 1] = px + timeStep * zpx
        if affine is not None:
            pxt[M - t - 1] += timeStep * (px @ affine[0][M - t - 1])
    return pxt, xt


def landmarkHamiltonianGradient(x0, at, px1, KparDiff, regweight, getCovector=False, affine=None):
    """pointEvolution.py:793-817: dat_k = 2 rw a_k - p_{k+1}."""
    pxt, xt = landmarkHamiltonianCovector(x0, at, px1, KparDiff, regweight, affine=affine)
    dat = 2 * regweight * at - pxt[1:]
    if getCovector:
        return dat, xt, pxt
    return dat, xt


# ---------------------------------------------------------------------------
# Surfaces (py-lddmm/surfaces.py)
# ---------------------------------------------------------------------------
class Surface:
    """Geometry subset of surfaces.Surface used on the hot path (surfaces.py:24-75, 261-263, 711-717)."""

    def __init__(self, surf=None, FV=None):
        if surf is not None:
            self.vertices = np.copy(surf.vertices)
            self.faces = np.copy(surf.faces)
        else:
            self.vertices = np.copy(FV[1])
            self.faces = np.int_(FV[0])
        self.computeCentersAreas()

    def computeCentersAreas(self):
        x1 = self.vertices[self.faces[:, 0]]
        x2 = self.vertices[self.faces[:, 1]]
        x3 = self.vertices[self.faces[:, 2]]
        self.centers = (x1 + x2 + x3) / 3
        self.surfel = np.cross(x2 - x1, x3 - x1)

    def updateVertices(self, x0):
        self.vertices = np.copy(x0)
        self.computeCentersAreas()

    def flipFaces(self):
        self.faces = self.faces[:, [0, 2, 1]]
        self.computeCentersAreas()

    def surfVolume(self):
        v = self.vertices[self.faces]
        return float((np.linalg.det(v) / 6).sum())


def _scatter3(fv, dz1, z1):
    """Vertex scatter of surfaces.py:1069-1089 (same for the three norms)."""
    x = fv.vertices
    F = fv.faces
    x1, x2, x3 = x[F[:, 0]], x[F[:, 1]], x[F[:, 2]]
    px = np.zeros(x.shape)
    np.add.at(px, F[:, 0], dz1 - np.cross(x3 - x2, z1))
    np.add.at(px, F[:, 1], dz1 - np.cross(x1 - x3, z1))
    np.add.at(px, F[:, 2], dz1 - np.cross(x2 - x1, z1))
    return 2 * px


def currentNorm0(fv1, KparDist):
    """surfaces.py:1009-1016."""
    return np.multiply(fv1.surfel, KparDist.applyK(fv1.centers, fv1.surfel)).sum()


def currentNormDef(fvDef, fv1, KparDist):
    """surfaces.py:1020-1033."""
    c1, cr1, c2, cr2 = fvDef.centers, fvDef.surfel, fv1.centers, fv1.surfel
    return (np.multiply(cr1, KparDist.applyK(c1, cr1)).sum()
            - 2 * np.multiply(cr1, KparDist.applyK(c2, cr2, firstVar=c1)).sum())


def currentNormGradient(fvDef, fv1, KparDist):
    """surfaces.py:1040-1089."""
    c1, cr1, c2, cr2 = fvDef.centers, fvDef.surfel, fv1.centers, fv1.surfel
    z1 = KparDist.applyK(c1, cr1) - KparDist.applyK(c2, cr2, firstVar=c1)
    dz1 = (1. / 3.) * (KparDist.applyDiffKT(c1, cr1[np.newaxis], cr1[np.newaxis])
                       - KparDist.applyDiffKT(c2, cr1[np.newaxis], cr2[np.newaxis], firstVar=c1))
    return _scatter3(fvDef, dz1, z1)


def measureNorm0(fv1, KparDist):
    """surfaces.py:1092-1099."""
    a2 = np.sqrt((fv1.surfel ** 2).sum(axis=1) + 1e-10)[:, np.newaxis]
    return np.multiply(a2, KparDist.applyK(fv1.centers, a2)).sum()


def measureNormDef(fvDef, fv1, KparDist):
    """surfaces.py:1104-1117."""
    a1 = np.sqrt((fvDef.surfel ** 2).sum(axis=1) + 1e-10)[:, np.newaxis]
    a2 = np.sqrt((fv1.surfel ** 2).sum(axis=1) + 1e-10)[:, np.newaxis]
    c1, c2 = fvDef.centers, fv1.centers
    return (np.multiply(a1, KparDist.applyK(c1, a1)).sum()
            - 2 * np.multiply(a1, KparDist.applyK(c2, a2, firstVar=c1)).sum())


def measureNormGradient(fvDef, fv1, KparDist):
    """surfaces.py:1125-1182."""
    c1, cr1, c2, cr2 = fvDef.centers, fvDef.surfel, fv1.centers, fv1.surfel
    a1 = np.sqrt((cr1 ** 2).sum(axis=1) + 1e-10)
    a2 = np.sqrt((cr2 ** 2).sum(axis=1) + 1e-10)
    n1 = cr1 / a1[:, np.newaxis]
    z1 = KparDist.applyK(c1, a1[:, np.newaxis]) - KparDist.applyK(c2, a2[:, np.newaxis], firstVar=c1)
    z1 = z1 * n1
    dz1 = (1. / 3.) * (KparDist.applyDiffKT(c1, a1[np.newaxis, :, np.newaxis], a1[np.newaxis, :, np.newaxis])
                       - KparDist.applyDiffKT(c2, a1[np.newaxis, :, np.newaxis], a2[np.newaxis, :, np.newaxis],
                                              firstVar=c1))
    return _scatter3(fvDef, dz1, z1)


def _varifold_terms(c1, cr1, c2, cr2):
    a1 = np.sqrt((cr1 ** 2).sum(axis=1) + 1e-10)
    a2 = np.sqrt((cr2 ** 2).sum(axis=1) + 1e-10)
    return a1, a2, cr1 / a1[:, np.newaxis], cr2 / a2[:, np.newaxis]


def varifoldNorm0(fv1, KparDist):
    """surfaces.py:1184-1196 (dense F x F weights, as the reference)."""
    _, a2, _, n2 = _varifold_terms(fv1.centers, fv1.surfel, fv1.centers, fv1.surfel)
    nn = n2 @ n2.T
    beta2 = (1 + nn ** 2) * (a2[:, None] * a2[None, :])
    return KparDist.applyK(fv1.centers, beta2[..., np.newaxis], matrixWeights=True).sum()


def varifoldNormDef(fvDef, fv1, KparDist):
    """surfaces.py:1200-1221."""
    c1, c2 = fvDef.centers, fv1.centers
    a1, a2, n1, n2 = _varifold_terms(c1, fvDef.surfel, c2, fv1.surfel)
    beta1 = (1 + (n1 @ n1.T) ** 2) * (a1[:, None] * a1[None, :])
    beta2 = (1 + (n1 @ n2.T) ** 2) * (a1[:, None] * a2[None, :])
    return (KparDist.applyK(c1, beta1[..., np.newaxis], matrixWeights=True).sum()
            - 2 * KparDist.applyK(c2, beta2[..., np.newaxis], firstVar=c1, matrixWeights=True).sum())


def varifoldNormGradient(fvDef, fv1, KparDist):
    """surfaces.py:1228-1276."""
    c1, c2 = fvDef.centers, fv1.centers
    a1, a2, n1, n2 = _varifold_terms(c1, fvDef.surfel, c2, fv1.surfel)
    n11 = n1 @ n1.T
    n12 = n1 @ n2.T
    beta1 = a1[:, None] * a1[None, :] * (1 + n11 ** 2)
    beta2 = a1[:, None] * a2[None, :] * (1 + n12 ** 2)
    u1 = (2 * n11[..., None] * n1[None] - (n11 ** 2)[..., None] * n1[:, None] + n1[:, None]) * a1[None, :, None]
    u2 = (2 * n12[..., None] * n2[None] - (n12 ** 2)[..., None] * n1[:, None] + n1[:, None]) * a2[None, :, None]
    z1 = KparDist.applyK(c1, u1, matrixWeights=True) - KparDist.applyK(c2, u2, firstVar=c1, matrixWeights=True)
    dz1 = (1. / 3.) * (KparDist.applyDiffKmat(c1, beta1) - KparDist.applyDiffKmat(c2, beta2, firstVar=c1))
    return _scatter3(fvDef, dz1, z1)


# The same three varifold functions with the F x F weights formed per pair in
# C (oracle.varifold_pairs) instead of as dense arrays, for face counts whose
# F x F x 3 FP64 temporaries do not fit in host memory (about 10 GB per array
# at 20,480 faces).  The sums are linear in the source weights a_l, so the
# S1 and S2 terms of surfaces.py:1200-1276 are one call over the stacked
# sources [c1; c2] with signed weights.
def _pair_sources(fvA, fvB, wB):
    a1, a2, n1, n2 = _varifold_terms(fvA.centers, fvA.surfel, fvB.centers, fvB.surfel)
    if fvB is fvA:
        return fvA.centers, n1, a1, fvA.centers, n1, a1
    return (fvA.centers, n1, a1, np.vstack([fvA.centers, fvB.centers]), np.vstack([n1, n2]),
            np.concatenate([a1, wB * a2]))


def varifoldNorm0_pairs(fv1, KparDist):
    """varifoldNorm0 (surfaces.py:1184-1196) per pair."""
    c1, n1, a1, c, n, a = _pair_sources(fv1, fv1, 1.0)
    val, _, _ = _o.varifold_pairs(c1, n1, a1, c, n, a, KparDist.sigma, KparDist.order, want=("val",))
    return float(val.sum())


def varifoldNormDef_pairs(fvDef, fv1, KparDist):
    """varifoldNormDef (surfaces.py:1200-1221) per pair: <S1,S1> - 2 <S1,S2>."""
    c1, n1, a1, c, n, a = _pair_sources(fvDef, fv1, -2.0)
    val, _, _ = _o.varifold_pairs(c1, n1, a1, c, n, a, KparDist.sigma, KparDist.order, want=("val",))
    return float(val.sum())


def varifoldNormGradient_pairs(fvDef, fv1, KparDist):
    """varifoldNormGradient (surfaces.py:1228-1276) per pair: z1 = K u1 - K u2,
    dz1 = (K'beta1 - K'beta2) / 3, then the vertex scatter."""
    c1, n1, a1, c, n, a = _pair_sources(fvDef, fv1, -1.0)
    _, z1, dz = _o.varifold_pairs(c1, n1, a1, c, n, a, KparDist.sigma, KparDist.order, want=("z", "dz"))
    return _scatter3(fvDef, (1. / 3.) * dz, z1)


# ---------------------------------------------------------------------------
# Curves (py-lddmm/curves.py)
# ---------------------------------------------------------------------------
class Curve:
    """Geometry subset of curves.Curve (curves.py:15-75)."""

    def __init__(self, curve=None, pointSet=None, FV=None, isOpen=False):
        if curve is not None:
            self.vertices = np.copy(curve.vertices)
            self.faces = np.copy(curve.faces)
        elif pointSet is not None:
            self.vertices = np.copy(pointSet)
            n = pointSet.shape[0]
            self.faces = np.int_(np.zeros([n, 2]))
            for k in range(n - 1):
                self.faces[k] = (k, k + 1)
            if not isOpen:
                self.faces[n - 1] = (n - 1, 0)
        else:
            self.vertices = np.copy(FV[1])
            self.faces = np.int_(FV[0])
        self.computeCentersLengths()

    def computeCentersLengths(self):
        x1 = self.vertices[self.faces[:, 0]]
        x2 = self.vertices[self.faces[:, 1]]
        self.centers = (x1 + x2) / 2
        self.lenel = x2 - x1

    def updateVertices(self, x0):
        self.vertices = np.copy(x0)
        self.computeCentersLengths()


def _scatter2(fv, dz1, z1):
    """curves.py:596-613."""
    px = np.zeros(fv.vertices.shape)
    np.add.at(px, fv.faces[:, 0], dz1 - z1)
    np.add.at(px, fv.faces[:, 1], dz1 + z1)
    return 2 * px


def curve_currentNorm0(fv1, KparDist):
    """curves.py:539-543."""
    return np.multiply(fv1.lenel, KparDist.applyK(fv1.centers, fv1.lenel)).sum()


def curve_currentNormDef(fvDef, fv1, KparDist):
    """curves.py:549-559."""
    c1, cr1, c2, cr2 = fvDef.centers, fvDef.lenel, fv1.centers, fv1.lenel
    return (np.multiply(cr1, KparDist.applyK(c1, cr1)).sum()
            - 2 * np.multiply(cr1, KparDist.applyK(c2, cr2, firstVar=c1)).sum())


def curve_currentNormGradient(fvDef, fv1, KparDist):
    """curves.py:566-613 (factor 1/2)."""
    c1, cr1, c2, cr2 = fvDef.centers, fvDef.lenel, fv1.centers, fv1.lenel
    z1 = KparDist.applyK(c1, cr1) - KparDist.applyK(c2, cr2, firstVar=c1)
    dz1 = .5 * (KparDist.applyDiffKT(c1, cr1[np.newaxis], cr1[np.newaxis])
                - KparDist.applyDiffKT(c2, cr1[np.newaxis], cr2[np.newaxis], firstVar=c1))
    return _scatter2(fvDef, dz1, z1)


def curve_measureNorm0(fv1, KparDist):
    """curves.py:621-627 -- no 1e-10 under the square root here (reference quirk)."""
    a2 = np.sqrt((fv1.lenel ** 2).sum(axis=1))[:, np.newaxis]
    return np.multiply(a2, KparDist.applyK(fv1.centers, a2)).sum()


def curve_measureNormDef(fvDef, fv1, KparDist):
    """curves.py:632-645."""
    a1 = np.sqrt((fvDef.lenel ** 2).sum(axis=1) + 1e-10)[:, np.newaxis]
    a2 = np.sqrt((fv1.lenel ** 2).sum(axis=1) + 1e-10)[:, np.newaxis]
    c1, c2 = fvDef.centers, fv1.centers
    return (np.multiply(a1, KparDist.applyK(c1, a1)).sum()
            - 2 * np.multiply(a1, KparDist.applyK(c2, a2, firstVar=c1)).sum())


def curve_measureNormGradient(fvDef, fv1, KparDist):
    """curves.py:653-703."""
    c1, cr1, c2, cr2 = fvDef.centers, fvDef.lenel, fv1.centers, fv1.lenel
    a1 = np.sqrt((cr1 ** 2).sum(axis=1) + 1e-10)
    a2 = np.sqrt((cr2 ** 2).sum(axis=1) + 1e-10)
    n1 = cr1 / a1[:, np.newaxis]
    z1 = (KparDist.applyK(c1, a1[:, np.newaxis]) - KparDist.applyK(c2, a2[:, np.newaxis], firstVar=c1)) * n1
    dz1 = (1. / 2.) * (KparDist.applyDiffKT(c1, a1[np.newaxis, :, np.newaxis], a1[np.newaxis, :, np.newaxis])
                       - KparDist.applyDiffKT(c2, a1[np.newaxis, :, np.newaxis], a2[np.newaxis, :, np.newaxis],
                                              firstVar=c1))
    return _scatter2(fvDef, dz1, z1)


# ---------------------------------------------------------------------------
# Optimisers (py-lddmm/conjugateGradient.py:33-217, gradientDescent.py:5-31)
# ---------------------------------------------------------------------------
def cg(opt, verb=True, maxIter=1000, TestGradient=False, epsInit=10., trace=None):
    """Polak-Ribiere+ nonlinear CG with the reference's line search
    (conjugateGradient.py:33-217).  ``trace`` (a list) receives the accepted
    objective after each iteration."""
    gradEps = getattr(opt, 'gradEps', 1.0)
    cgBurnIn = getattr(opt, 'cgBurnIn', -1)
    gradCoeff = getattr(opt, 'gradCoeff', 1.0)
    restartRate = getattr(opt, 'restartRate', 100)
    eps = epsInit
    epsMin = 1e-10
    opt.converged = False
    obj = opt.objectiveFun()
    skipCG = 0
    for it in range(maxIter):
        if it % restartRate == 0:
            skipCG = 1
        grd = opt.getGradient(gradCoeff)
        if TestGradient:
            dirfoo = opt.randomDir()
            epsfoo = 1e-7
            objfoo = opt.updateTry(dirfoo, epsfoo, obj - 1e10)
            [grdfoo] = opt.dotProduct(grd, [dirfoo])
            logging.info('Test Gradient: %.4f %.4f' % ((objfoo - obj) / epsfoo, -grdfoo * gradCoeff))
        if it == 0 or it == cgBurnIn:
            [grdOld2] = opt.dotProduct(grd, [grd])
            grd2 = grdOld2
            grdTry = np.sqrt(max(1e-20, grdOld2))
            oldDir = opt.copyDir(grd)
            grdOld = opt.copyDir(grd)
            dir0 = opt.copyDir(grd)
            beta = 0
        else:
            [grd2, grd12] = opt.dotProduct(grd, [grd, grdOld])
            beta = max(0, (grd2 - grd12) / grdOld2) if skipCG == 0 else 0
            grdOld2 = grd2
            grdTry = np.sqrt(max(1e-20, grd2 + beta * grd12))
            dir0 = opt.addProd(grd, oldDir, beta)
            oldDir = opt.copyDir(dir0)
            grdOld = opt.copyDir(grd)
        objTry = opt.updateTry(dir0, eps, obj)
        noUpdate = 0
        if objTry > obj:
            epsSmall = 0.000001 / grdTry
            objTry0 = opt.updateTry(dir0, epsSmall, obj)
            if objTry0 > obj:
                if (skipCG == 1) | (beta < 1e-10):
                    logging.info('Stopping Gradient Descent: bad direction')
                    break
                elif verb:
                    # conjugateGradient.py:151-154: only under `if verb:`
                    skipCG = 1
                    noUpdate = 1
            else:
                while (objTry > obj) and (eps > epsMin):
                    eps = eps / 2
                    objTry = opt.updateTry(dir0, eps, obj)
        if noUpdate == 0:
            contt = 1
            while contt == 1:
                objTry2 = opt.updateTry(dir0, .5 * eps, objTry)
                if objTry > objTry2:
                    eps = eps / 2
                    objTry = objTry2
                else:
                    contt = 0
            contt = 1
            while contt == 1:
                objTry2 = opt.updateTry(dir0, 1.25 * eps, objTry)
                if objTry > objTry2:
                    eps *= 1.25
                    objTry = objTry2
                else:
                    contt = 0
            if np.fabs(obj - objTry) < .000001:
                if (skipCG == 1) | (beta < 1e-10):
                    opt.converged = True
                    break
                else:
                    skipCG = 1
                    eps = 1.0
            else:
                skipCG = 0
            opt.acceptVarTry()
            obj = objTry
            if trace is not None:
                trace.append(obj)
            if np.sqrt(grd2) < gradEps:
                opt.converged = True
                break
            eps = 100 * eps
            if hasattr(opt, 'endOfIteration'):
                opt.endOfIteration()
    if hasattr(opt, 'endOptim'):
        opt.endOptim()
    return opt.getVariable()


def descend(opt, verb=True, maxIter=1000, TestGradient=False, epsInit=10., trace=None):
    """gradientDescent.py:5-31."""
    eps = epsInit
    gradCoeff = 1.0
    obj = opt.objectiveFun()
    for it in range(maxIter):
        grd = opt.getGradient(gradCoeff)
        if (it % 10) == 0:
            eps *= 2.
        objTry = 1e30
        while objTry > obj and eps > 1e-20:
            objTry = opt.updateTry(grd, eps, obj)
            eps *= .5
        opt.acceptVarTry()
        obj = objTry
        if trace is not None:
            trace.append(obj)
        if hasattr(opt, 'endOfIteration'):
            opt.endOfIteration()


# ---------------------------------------------------------------------------
# Matching problems (surfaceMatching.py, curveMatching.py), affine 'none'
# ---------------------------------------------------------------------------
class Direction:
    def __init__(self):
        self.diff = []
        self.aff = []
        self.initx = []


class _MatchingBase:
    def _obj_def(self, at, withTrajectory=False):
        """objectiveFunDef (surfaceMatching.py:187-221 / curveMatching.py:148-182)."""
        timeStep = 1.0 / self.Tsize
        xt = landmarkDirectEvolutionEuler(self.x0, at, self.param.KparDiff)
        obj = 0
        for t in range(self.Tsize):
            ra = self.param.KparDiff.applyK(xt[t], at[t])
            obj = obj + self.regweight * timeStep * np.multiply(at[t], ra).sum()
        if withTrajectory:
            return obj, xt
        return obj

    def objectiveFun(self):
        if self.obj is None:
            self.obj0 = self.param.fun_obj0(self.fv1, self.param.KparDist) / (self.param.sigmaError ** 2)
            self.obj, self.xt = self._obj_def(self.at, withTrajectory=True)
            self.fvDef.updateVertices(self.xt[-1])
            self.obj += self.obj0 + self.dataTerm(self.fvDef)
        return self.obj

    def dataTerm(self, fvDef):
        return self.param.fun_obj(fvDef, self.fv1, self.param.KparDist) / (self.param.sigmaError ** 2)

    def getVariable(self):
        return [self.at]

    def updateTry(self, dir, eps, objRef=None):
        """surfaceMatching.py:255-289."""
        objTry = self.obj0
        atTry = self.at - eps * dir.diff
        foo = self._obj_def(atTry, withTrajectory=True)
        objTry += foo[0]
        ff = self._copy_shape(self.fvDef)
        ff.updateVertices(foo[1][-1])
        objTry += self.dataTerm(ff)
        if np.isnan(objTry):
            return 1e500
        if (objRef is None) or (objTry < objRef):
            self.atTry = atTry
            self.objTry = objTry
        return objTry

    def getGradient(self, coeff=1.0):
        """surfaceMatching.py:301-327."""
        px1 = -self.param.fun_objGrad(self.fvDef, self.fv1, self.param.KparDist) / self.param.sigmaError ** 2
        dat, _ = landmarkHamiltonianGradient(self.x0, self.at, px1, self.param.KparDiff, self.regweight)
        grd = Direction()
        grd.diff = dat / (coeff * self.Tsize)
        return grd

    def addProd(self, dir1, dir2, beta):
        d = Direction()
        d.diff = dir1.diff + beta * dir2.diff
        return d

    def copyDir(self, dir0):
        d = Direction()
        d.diff = np.copy(dir0.diff)
        return d

    def randomDir(self):
        d = Direction()
        d.diff = self.rng.standard_normal((self.Tsize, self.npt, self.dim))
        return d

    def dotProduct(self, g1, g2):
        """surfaceMatching.py:353-377."""
        res = np.zeros(len(g2))
        for t in range(self.Tsize):
            u = self.param.KparDiff.applyK(self.xt[t], g1.diff[t])
            for ll, gr in enumerate(g2):
                res[ll] = res[ll] + np.multiply(gr.diff[t], u).sum()
        return res

    def acceptVarTry(self):
        self.obj = self.objTry
        self.at = np.copy(self.atTry)

    def endOfIteration(self):
        self.iter += 1
        _, self.xt = self._obj_def(self.at, withTrajectory=True)
        self.fvDef.updateVertices(self.xt[-1])


class MatchingParam:
    """SurfaceMatchingParam / CurveMatchingParam (surfaceMatching.py:19-50, curveMatching.py:19-35)."""

    def __init__(self, timeStep=.1, KparDiff=None, KparDist=None, sigmaKernel=6.5, sigmaDist=2.5, sigmaError=1.0,
                 errorType='measure', typeKernel='gauss', curves=False):
        self.timeStep = timeStep
        self.sigmaError = sigmaError
        self.errorType = errorType
        table = {
            False: {'current': (currentNorm0, currentNormDef, currentNormGradient),
                    'measure': (measureNorm0, measureNormDef, measureNormGradient),
                    'varifold': (varifoldNorm0, varifoldNormDef, varifoldNormGradient)},
            True: {'current': (curve_currentNorm0, curve_currentNormDef, curve_currentNormGradient),
                   'measure': (curve_measureNorm0, curve_measureNormDef, curve_measureNormGradient)},
        }[curves]
        self.fun_obj0, self.fun_obj, self.fun_objGrad = table[errorType]
        self.KparDiff = KparDiff if KparDiff is not None else Kernel(name=typeKernel, sigma=sigmaKernel)
        self.KparDist = KparDist if KparDist is not None else Kernel(name='gauss', sigma=sigmaDist)


class SurfaceMatching(_MatchingBase):
    """surfaceMatching.py:74-484 with affine='none', symmetric=False, no file output."""

    def __init__(self, Template, Target, param, maxIter=1000, regWeight=1.0, testGradient=False, seed=0,
                 verb=True):
        self.verb = verb
        self.fv0 = Surface(surf=Template)
        self.fv1 = Surface(surf=Target)
        self.param = param
        if self.fv0.surfVolume() * self.fv1.surfVolume() < 0:   # surfaceMatching.py:126-129
            self.fv1.flipFaces()
        self.x0 = np.copy(self.fv0.vertices)
        self.fvDef = Surface(surf=self.fv0)
        self.npt = self.x0.shape[0]
        self.dim = self.x0.shape[1]
        self.maxIter = maxIter
        self.testGradient = testGradient
        self.regweight = regWeight
        self.Tsize = int(round(1.0 / param.timeStep))
        self.at = np.zeros([self.Tsize, self.npt, self.dim])
        self.atTry = np.zeros_like(self.at)
        self.xt = np.tile(self.x0, [self.Tsize + 1, 1, 1])
        self.obj = None
        self.objTry = None
        self.gradCoeff = self.npt
        self.iter = 0
        self.rng = np.random.default_rng(seed)

    @staticmethod
    def _copy_shape(s):
        return Surface(surf=s)

    def optimizeMatching(self, trace=None):
        """surfaceMatching.py:474-484."""
        grd = self.getGradient(self.gradCoeff)
        [grd2] = self.dotProduct(grd, [grd])
        self.gradEps = max(0.001, np.sqrt(grd2) / 10000)
        cg(self, verb=self.verb, maxIter=self.maxIter, TestGradient=self.testGradient, epsInit=0.1, trace=trace)


class CurveMatching(_MatchingBase):
    """curveMatching.py:58-352 with affine='none', no file output."""

    def __init__(self, Template, Target, param, maxIter=1000, regWeight=1.0, gradLB=0.001, testGradient=False,
                 seed=0, verb=True):
        self.verb = verb
        self.fv0 = Curve(curve=Template)
        self.fv1 = Curve(curve=Target)
        self.param = param
        self.x0 = self.fv0.vertices
        self.fvDef = Curve(curve=self.fv0)
        self.npt, self.dim = self.x0.shape
        self.maxIter = maxIter
        self.testGradient = testGradient
        self.regweight = regWeight
        self.Tsize = int(round(1.0 / param.timeStep))
        self.at = np.zeros([self.Tsize, self.npt, self.dim])
        self.atTry = np.zeros_like(self.at)
        self.xt = np.tile(self.x0, [self.Tsize + 1, 1, 1])
        self.obj = None
        self.objTry = None
        self.gradCoeff = self.npt
        self.gradLB = gradLB
        self.iter = 0
        self.rng = np.random.default_rng(seed)

    @staticmethod
    def _copy_shape(c):
        return Curve(curve=c)

    def optimizeMatching(self, trace=None, optimizer='cg'):
        """curveMatching.py:342-352 (cg with its default epsInit=10)."""
        grd = self.getGradient(self.gradCoeff)
        [grd2] = self.dotProduct(grd, [grd])
        self.gradEps = max(self.gradLB, np.sqrt(grd2) / 10000)
        if optimizer == 'cg':
            cg(self, verb=self.verb, maxIter=self.maxIter, TestGradient=self.testGradient, trace=trace)
        else:
            descend(self, verb=self.verb, maxIter=self.maxIter, trace=trace)


# ---------------------------------------------------------------------------
# Template estimation (py-lddmm/surfaceTemplate.py:33-369), affine 'none'
# ---------------------------------------------------------------------------
class TemplateDirection:
    """surfaceTemplate.py:13-16: `prior` (T, N, d) and one Direction per subject in `all`."""

    def __init__(self):
        self.prior = []
        self.all = []


class SurfaceTemplate:
    """surfaceTemplate.py:33-369 with affine='none' and no file output.

    The hyper-template fv0 is deformed by the prior momenta `at` into the
    template fvTmpl; the template is deformed by atAll[k] towards subject k.
    Objective (surfaceTemplate.py:170-190):
        sum_k Norm0(S_k)/s^2 + lambdaPrior E(at) + sum_k [E(atAll[k]) + NormDef(phi_k(Tmpl), S_k)/s^2].
    The reference's SurfaceTemplate inherits objectiveFunDef from
    SurfaceMatching but sets neither `x0` (read when no x0 is passed: the prior
    shot) nor `v` (a per-step velocity store): the hyper-template's vertices
    are the x0 of the prior shot here, and no velocity is stored."""

    def __init__(self, HyperTmpl, Targets, param, maxIter=1000, lambdaPrior=1.0, regWeight=1.0, testGradient=True,
                 seed=0, verb=True):
        self.verb = verb
        self.fv0 = Surface(surf=HyperTmpl)
        self.fv1 = [Surface(surf=ff) for ff in Targets]
        self.Ntarg = len(self.fv1)
        self.npt, self.dim = self.fv0.vertices.shape
        self.fvTmpl = Surface(surf=self.fv0)
        self.param = param
        self.maxIter = maxIter
        self.testGradient = testGradient
        self.regweight = regWeight
        self.lambdaPrior = lambdaPrior
        self.Tsize = int(round(1.0 / param.timeStep))
        shp = (self.Tsize, self.npt, self.dim)
        self.at = np.zeros(shp)
        self.atTry = np.zeros(shp)
        self.xt = np.tile(self.fv0.vertices, [self.Tsize + 1, 1, 1])
        self.atAll = [np.zeros(shp) for _ in self.fv1]
        self.atAllTry = [np.zeros(shp) for _ in self.fv1]
        self.xtAll = [np.tile(self.fv0.vertices, [self.Tsize + 1, 1, 1]) for _ in self.fv1]
        self.fvDef = [Surface(surf=self.fv0) for _ in self.fv1]
        self.tmplCoeff = 1.0
        self.obj = None
        self.objTry = None
        self.gradCoeff = self.npt
        self.iter = 0
        self.rng = np.random.default_rng(seed)

    def _obj_def(self, at, x0):
        """objectiveFunDef (surfaceMatching.py:187-221) from x0."""
        timeStep = 1.0 / self.Tsize
        xt = landmarkDirectEvolutionEuler(x0, at, self.param.KparDiff)
        obj = 0
        for t in range(self.Tsize):
            ra = self.param.KparDiff.applyK(xt[t], at[t])
            obj = obj + self.regweight * timeStep * np.multiply(at[t], ra).sum()
        return obj, xt

    def _data(self, x, kk):
        ff = Surface(surf=self.fv0)
        ff.updateVertices(x)
        return self.param.fun_obj(ff, self.fv1[kk], self.param.KparDist) / (self.param.sigmaError ** 2)

    def objectiveFun(self):
        """surfaceTemplate.py:170-190."""
        if self.obj is None:
            self.obj0 = 0
            for fv in self.fv1:
                self.obj0 += self.param.fun_obj0(fv, self.param.KparDist) / (self.param.sigmaError ** 2)
            self.obj = self.obj0
            e, self.xt = self._obj_def(self.at, self.fv0.vertices)
            self.fvTmpl.updateVertices(self.xt[-1])
            self.obj += e * self.lambdaPrior
            for kk, a in enumerate(self.atAll):
                e, xk = self._obj_def(a, self.fvTmpl.vertices)
                self.obj += e + self._data(xk[-1], kk)
                self.xtAll[kk] = np.copy(xk)
        return self.obj

    def getVariable(self):
        return self.fvTmpl

    def copyDir(self, dir0):
        d = TemplateDirection()
        d.prior = np.copy(dir0.prior)
        for g in dir0.all:
            d.all.append(Direction())
            d.all[-1].diff = np.copy(g.diff)
        return d

    def randomDir(self):
        d = TemplateDirection()
        d.prior = self.rng.standard_normal((self.Tsize, self.npt, self.dim))
        for _ in range(self.Ntarg):
            d.all.append(Direction())
            d.all[-1].diff = self.rng.standard_normal((self.Tsize, self.npt, self.dim))
        return d

    def updateTry(self, dir, eps, objRef=None):
        """surfaceTemplate.py:215-238."""
        objTry = self.obj0
        atTry = self.at - eps * dir.prior
        e, xt = self._obj_def(atTry, self.fv0.vertices)
        objTry += e * self.lambdaPrior
        x0 = xt[-1]
        atAllTry = []
        for kk, d in enumerate(dir.all):
            atAllTry.append(self.atAll[kk] - eps * d.diff)
            e, xk = self._obj_def(atAllTry[kk], x0)
            objTry += e + self._data(xk[-1], kk)
        if (objRef is None) or (objTry < objRef):
            self.atTry = atTry
            self.atAllTry = atAllTry
            self.objTry = objTry
        return objTry

    def getGradient(self, coeff=1.0):
        """surfaceTemplate.py:241-301: per subject the Hamiltonian gradient from
        the template, its covector at t = 0 summed into the template's end-point
        covector, then the prior's gradient from the hyper-template."""
        pxTmpl = np.zeros((self.npt, self.dim))
        grd = TemplateDirection()
        for kk in range(self.Ntarg):
            px1 = -self.param.fun_objGrad(self.fvDef[kk], self.fv1[kk], self.param.KparDist) / \
                self.param.sigmaError ** 2
            dat, _, pxt = landmarkHamiltonianGradient(self.fvTmpl.vertices, self.atAll[kk], px1, self.param.KparDiff,
                                                      self.regweight, getCovector=True)
            grd.all.append(Direction())
            grd.all[kk].diff = dat / (coeff * self.Tsize)
            pxTmpl += pxt[0]
        dat, _ = landmarkHamiltonianGradient(self.fv0.vertices, self.at, pxTmpl / self.lambdaPrior,
                                             self.param.KparDiff, self.regweight)
        grd.prior = dat / (self.tmplCoeff * coeff * self.Tsize)
        return grd

    def dotProduct(self, g1, g2):
        """surfaceTemplate.py:303-334."""
        res = np.zeros(len(g2))
        for kk, gg1 in enumerate(g1.all):
            for t in range(self.Tsize):
                u = self.param.KparDiff.applyK(self.xtAll[kk][t], gg1.diff[t])
                for ll, gr in enumerate(g2):
                    res[ll] = res[ll] + np.multiply(gr.all[kk].diff[t], u).sum()
        for t in range(g1.prior.shape[0]):
            u = self.param.KparDiff.applyK(self.xt[t], g1.prior[t])
            for ll, gr in enumerate(g2):
                res[ll] = res[ll] + np.multiply(gr.prior[t], u).sum() * (self.tmplCoeff * self.lambdaPrior)
        return res

    def acceptVarTry(self):
        self.obj = self.objTry
        self.at = np.copy(self.atTry)
        for kk, a in enumerate(self.atAllTry):
            self.atAll[kk] = np.copy(a)

    def addProd(self, dir1, dir2, coeff):
        res = TemplateDirection()
        res.prior = dir1.prior + coeff * dir2.prior
        for kk, dd in enumerate(dir1.all):
            res.all.append(Direction())
            res.all[kk].diff = dd.diff + coeff * dir2.all[kk].diff
        return res

    def endOfIteration(self):
        """surfaceTemplate.py:353-361 without the VTK output."""
        self.iter += 1
        _, self.xt = self._obj_def(self.at, self.fv0.vertices)
        self.fvTmpl.updateVertices(self.xt[-1])
        for kk in range(self.Ntarg):
            _, self.xtAll[kk] = self._obj_def(self.atAll[kk], self.xt[-1])
            self.fvDef[kk].updateVertices(self.xtAll[kk][-1])

    def computeTemplate(self, trace=None):
        """surfaceTemplate.py:363-369: gradEps = max(0.1, |g|/1e4); cg with
        TestGradient=True and the default epsInit."""
        grd = self.getGradient(self.gradCoeff)
        [grd2] = self.dotProduct(grd, [grd])
        self.gradEps = max(0.1, np.sqrt(grd2) / 10000)
        cg(self, verb=self.verb, maxIter=self.maxIter, TestGradient=self.testGradient, trace=trace)
        return self
