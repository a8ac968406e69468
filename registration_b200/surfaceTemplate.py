"""Surface template estimation with the interface of py-lddmm/surfaceTemplate.py, on the GPU.

  SurfaceTemplate(HyperTmpl, Targets, ..., param, maxIter, lambdaPrior, regWeight, ...)    surfaceTemplate.py:33-123
      .computeTemplate()                                                               surfaceTemplate.py:363-369

The hyper-template fv0 is deformed by the prior momenta `at` into the template
fvTmpl; the template is deformed by atAll[k] towards every subject k.  The
objective (surfaceTemplate.py:170-190) is

    sum_k Norm0(S_k)/s^2 + lambdaPrior E(at) + sum_k [E(atAll[k]) + NormDef(phi_k(Tmpl), S_k)/s^2],

E the deformation energy rw dt sum_t <a_t, K(x_t) a_t>.  The subjects'
problems are independent given the template, so each evaluation runs them as
ONE ragged launch per kernel family (lddmm_ragged_shoot / _dataterm /
_covector / _applyk: one segment per subject), and the prior as one
single-problem shot / adjoint.  Momenta, trajectories and directions stay on
the device ((K, T, N, d) tensors; atAll[k] indexes like the reference's list);
each objective value and dot product is one host read.

Kernel sums run in KparDiff's precision: FP32 compensated ('fp32c', the
ragged path) or FP64 (the subjects are then looped over with the FP64
single-problem kernels).  lineSearchPrecision ('fp64' default, 'auto',
'fp32c') selects the data-term values the line search compares, as for
SurfaceMatching.

The reference's SurfaceTemplate inherits objectiveFunDef from SurfaceMatching
but sets neither `x0` (read by the prior's shot, which passes no x0) nor `v`
(a velocity store); here the prior shot starts from the hyper-template's
vertices, the only value those calls can mean.  Only affine='none' is
provided; VTK output of the iterates is not written.
"""
import logging

import numpy as np
import torch

from . import _ragged as _rg
from . import conjugateGradient as cg
from . import pointEvolution as evol
from . import surfaceMatching as smatch
from . import surfaces
from ._precision import _Value, value_bound
from .device import require_cuda, to_dev


class Direction:
    """surfaceTemplate.py:13-16.  `prior` (T, N, d); the subjects' directions
    are one (K, T, N, d) tensor `stack`; `all[k].diff` is a view of stack[k]."""

    def __init__(self, prior=None, stack=None):
        self.prior = prior
        self.stack = stack

    @property
    def all(self):
        out = []
        for k in range(self.stack.shape[0]):
            d = smatch.Direction()
            d.diff = self.stack[k]
            d.aff = np.zeros((self.stack.shape[1], 0))
            out.append(d)
        return out


class SurfaceTemplate:
    def __init__(self, HyperTmpl=None, Targets=None, fileHTempl=None, fileTarg=None, param=None, maxIter=1000,
                 lambdaPrior=1.0, regWeight=1.0, affineWeight=1.0, verb=True, rotWeight=None, scaleWeight=None,
                 transWeight=None, testGradient=False, saveFile='evolution', affine='none', outputDir='.',
                 lineSearchPrecision='fp64', noise=1e-8):
        require_cuda()
        if HyperTmpl is None:
            if fileHTempl is None:
                raise ValueError('Please provide a hyper-template surface')
            HyperTmpl = surfaces.Surface(filename=fileHTempl)
        if Targets is None:
            if fileTarg is None:
                raise ValueError('Please provide target surfaces')
            Targets = [surfaces.Surface(filename=ff) for ff in fileTarg]
        if affine not in ('none', None):
            raise NotImplementedError("affine registration components are not provided (affine='none' only)")
        if lineSearchPrecision not in ('fp64', 'auto', 'fp32c'):
            raise ValueError("lineSearchPrecision must be 'fp64', 'auto' or 'fp32c'")
        self.fv0 = surfaces.Surface(surf=HyperTmpl)
        self.fv1 = [surfaces.Surface(surf=ff) for ff in Targets]
        if not self.fv1:
            raise ValueError('Please provide Target surfaces')
        self.Ntarg = len(self.fv1)
        self.param = param if param is not None else smatch.SurfaceMatchingParam()
        if self.param.errorType not in _rg.NORMS:
            raise ValueError("errorType must be one of %s" % sorted(_rg.NORMS))
        self.saveFile = saveFile
        self.outputDir = outputDir
        self.maxIter = maxIter
        self.verb = verb
        self.testGradient = testGradient
        self.regweight = regWeight
        self.lambdaPrior = lambdaPrior
        self.affine = 'none'
        self.affineDim = 0
        self.tmplCoeff = 1.0
        self.Tsize = int(round(1.0 / self.param.timeStep))
        self.x0 = to_dev(self.fv0.vertices)
        self.npt, self.dim = self.x0.shape
        dev = self.x0.device
        T, N, d, K = self.Tsize, self.npt, self.dim, self.Ntarg
        self.fvTmpl = surfaces.Surface(surf=self.fv0)
        self.fvDef = [surfaces.Surface(surf=self.fv0) for _ in range(K)]
        self.at = torch.zeros((T, N, d), dtype=torch.float64, device=dev)
        self.atTry = self.at
        self.atAll = torch.zeros((K, T, N, d), dtype=torch.float64, device=dev)
        self.atAllTry = self.atAll
        self.Afft = np.zeros((T, 0))
        self.AfftAll = [np.zeros((T, 0)) for _ in range(K)]
        self.xt = self.x0.unsqueeze(0).repeat(T + 1, 1, 1)
        self.xtAll = self.x0.expand(K, T + 1, N, d).clone()
        self._try = None
        self.obj = None
        self.objTry = None
        self.gradCoeff = self.npt
        self.iter = 0
        self.calls = {"updateTry": 0, "getGradient": 0, "dotProduct": 0, "refine": 0}
        # device topology of the template (shared by every subject's deformed template) and targets
        self._dshape = self.fv0.device_shape()
        self._tc = [to_dev(f.centers) for f in self.fv1]
        self._tv = [to_dev(f.surfel) for f in self.fv1]
        self._s2 = float(self.param.sigmaError) ** 2
        Kd = self.param.KparDiff
        self._ragged = Kd.precision == 'fp32c'
        self._ord_diff = _rg.kernel_order(Kd)
        self._ord_dist = _rg.kernel_order(self.param.KparDist)
        self._auto = lineSearchPrecision == 'auto'
        self._noise = float(noise)
        self.noise_obs = 0.0
        self._val_prec = self.param.KparDist.precision if self._auto else lineSearchPrecision
        self._grad_prec = self.param.KparDist.precision

    # -- building blocks -----------------------------------------------------------------
    def _shoot_prior(self, at):
        return evol.shoot(self.x0, at, self.param.KparDiff, regweight=self.regweight, with_energy=True)

    def _shoot_subjects(self, x_tmpl, atAll):
        """Every subject's shot from the template: (K, T+1, N, d) and energies (K,)."""
        K, T, N, d = atAll.shape
        if self._ragged:
            v_off = [k * N for k in range(K + 1)]
            XT, E = _rg.shoot(x_tmpl.repeat(K, 1), atAll.reshape(-1, d), v_off, T, [self.param.KparDiff.sigma] * K,
                              self._ord_diff, [self.regweight] * K)
            return XT.view(K, T + 1, N, d), E
        xs, es = [], []
        for k in range(K):
            xk, ek = evol.shoot(x_tmpl, atAll[k], self.param.KparDiff, regweight=self.regweight, with_energy=True)
            xs.append(xk)
            es.append(ek.reshape(1))
        return torch.stack(xs), torch.cat(es)

    def _data_values(self, ends, precision):
        """NormDef(phi_k(Tmpl), S_k) of every subject (one ragged launch), (K,)."""
        K = len(ends)
        return _rg.dataterm(self.param.errorType, list(ends), [self._dshape] * K, self._tc, self._tv,
                            [self.param.KparDist.sigma] * K, self._ord_dist, precision, grad=False)

    def _value(self, at, atAll):
        xt, e0 = self._shoot_prior(at)
        xall, ek = self._shoot_subjects(xt[-1], atAll)
        D = self._data_values(xall[:, -1], self._val_prec)
        host = torch.stack([e0.reshape(()) * self.lambdaPrior + ek.sum(), (D / self._s2).sum()]).cpu().numpy()
        ereg, data = float(host[0]), float(host[1])
        v = self.obj0 + ereg + data
        if self._auto:
            v = _Value(v, self, ereg, xall[:, -1], value_bound(self, self._noise, self.obj0))
        return v, xt, xall

    def exact_value(self, ereg, x_end):
        """The objective with FP64 data-term values (refinement of a _Value)."""
        self.calls["refine"] += 1
        return self.obj0 + ereg + float((self._data_values(x_end, 'fp64') / self._s2).sum())

    # -- optimiser protocol (conjugateGradient.cg) ----------------------------------------
    def objectiveFun(self):
        """surfaceTemplate.py:170-190."""
        if self.obj is None:
            K = self.Ntarg
            prec = 'fp64' if self._auto else self._val_prec
            norm0 = _rg.dataterm(self.param.errorType, [to_dev(f.vertices) for f in self.fv1],
                                 [f.device_shape() for f in self.fv1], None, None,
                                 [self.param.KparDist.sigma] * K, self._ord_dist, prec, grad=False)
            self.obj0 = float((norm0 / self._s2).sum())
            self.obj, self.xt, self.xtAll = self._value(self.at, self.atAll)
            self.fvTmpl.updateVertices(self.xt[-1])
        return self.obj

    def getVariable(self):
        return self.fvTmpl

    def copyDir(self, dir0):
        return Direction(dir0.prior.clone(), dir0.stack.clone())

    def randomDir(self):
        return Direction(torch.randn_like(self.at), torch.randn_like(self.atAll))

    def addProd(self, dir1, dir2, coeff):
        return Direction(dir1.prior + coeff * dir2.prior, dir1.stack + coeff * dir2.stack)

    def updateTry(self, dir, eps, objRef=None):
        """surfaceTemplate.py:215-238; NaN objectives return 1e500."""
        self.calls["updateTry"] += 1
        atTry = self.at - eps * dir.prior
        atAllTry = self.atAll - eps * dir.stack
        objTry, xt, xall = self._value(atTry, atAllTry)
        if np.isnan(objTry):
            logging.info('Warning: nan in updateTry')
            return 1e500
        if (objRef is None) or (objTry < objRef):
            self.atTry = atTry
            self.atAllTry = atAllTry
            self.objTry = objTry
            self._try = (xt, xall)
        return objTry

    def getGradient(self, coeff=1.0):
        """surfaceTemplate.py:241-301: every subject's Hamiltonian gradient from the
        template (one ragged adjoint), their covectors at t = 0 summed into the
        template's end-point covector, then the prior's gradient."""
        self.calls["getGradient"] += 1
        K, T, N, d = self.atAll.shape
        pxs = _rg.dataterm(self.param.errorType, list(self.xtAll[:, -1]), [self._dshape] * K, self._tc, self._tv,
                           [self.param.KparDist.sigma] * K, self._ord_dist, self._grad_prec, grad=True)
        px1 = torch.stack(pxs) / (-self._s2)
        if self._ragged:
            v_off = [k * N for k in range(K + 1)]
            pxt, dat = _rg.covector(self.xtAll.reshape(-1, d), self.atAll.reshape(-1, d), px1.reshape(-1, d), v_off,
                                    T, [self.param.KparDiff.sigma] * K, self._ord_diff, [self.regweight] * K)
            pxt = pxt.view(K, T + 1, N, d)
            dat = dat.view(K, T, N, d)
        else:
            outs = [evol.covector(self.xtAll[k], self.atAll[k], px1[k], self.param.KparDiff, self.regweight,
                                  with_dat=True) for k in range(K)]
            pxt = torch.stack([o[0] for o in outs])
            dat = torch.stack([o[1] for o in outs])
        pxTmpl = pxt[:, 0].sum(dim=0)
        _, dat0 = evol.covector(self.xt, self.at, pxTmpl / self.lambdaPrior, self.param.KparDiff, self.regweight,
                                with_dat=True)
        return Direction(dat0 / (self.tmplCoeff * coeff * T), dat / (coeff * T))

    def dotProduct(self, g1, g2):
        """surfaceTemplate.py:303-334: sum_k sum_t <g2_kt, K(x_kt) g1_kt>
        + tmplCoeff lambdaPrior sum_t <g2_t, K(x_t) g1_t>, one ragged applyK
        over the K T + T segments, FP64 reductions, one host read."""
        self.calls["dotProduct"] += 1
        K, T, N, d = self.atAll.shape
        if self._ragged:
            X = torch.cat([self.xtAll[:, :T].reshape(-1, d), self.xt[:T].reshape(-1, d)])
            G = torch.cat([g1.stack.reshape(-1, d), g1.prior.reshape(-1, d)])
            starts = [s * N for s in range(K * T + T)]
            U = _rg.applyk_segments(X, G, starts, [N] * (K * T + T), [self.param.KparDiff.sigma] * (K * T + T),
                                    self._ord_diff)
            u_all, u_prior = U[:K * T * N].reshape(-1), U[K * T * N:].reshape(-1)
        else:
            Kd = self.param.KparDiff
            u_all = torch.stack([torch.stack([Kd.applyK(self.xtAll[k, t], g1.stack[k, t]) for t in range(T)])
                                 for k in range(K)]).reshape(-1)
            u_prior = torch.stack([Kd.applyK(self.xt[t], g1.prior[t]) for t in range(T)]).reshape(-1)
        G2a = torch.stack([g.stack.reshape(-1) for g in g2])
        G2p = torch.stack([g.prior.reshape(-1) for g in g2])
        res = G2a @ u_all + (G2p @ u_prior) * (self.tmplCoeff * self.lambdaPrior)
        return res.cpu().numpy()

    def acceptVarTry(self):
        self.obj = self.objTry
        self.at = self.atTry.clone()
        self.atAll = self.atAllTry.clone()
        if self._try is not None:
            self.xt, self.xtAll = self._try

    def endOfIteration(self):
        """surfaceTemplate.py:353-361 without the VTK output; the accepted trial's
        trajectories are kept (re-shooting would reproduce them bit for bit)."""
        self.iter += 1
        self.fvTmpl.updateVertices(self.xt[-1])
        for k in range(self.Ntarg):
            self.fvDef[k].updateVertices(self.xtAll[k, -1])

    def endOptim(self):
        if isinstance(self.obj, _Value):
            self.obj = float(self.obj.refine())

    def computeTemplate(self, testGradient=True):
        """surfaceTemplate.py:363-369: gradEps = max(0.1, |g|/1e4), then cg with its
        default epsInit.  The reference always passes TestGradient=True (one
        random-direction trial per iteration that only logs a check and leaves
        the iterates unchanged); testGradient=False skips it."""
        grd = self.getGradient(self.gradCoeff)
        [grd2] = self.dotProduct(grd, [grd])
        self.gradEps = max(0.1, np.sqrt(grd2) / 10000)
        cg.cg(self, verb=self.verb, maxIter=self.maxIter, TestGradient=testGradient)
        return self
