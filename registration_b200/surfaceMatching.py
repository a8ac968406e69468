"""Surface matching with the interface of py-lddmm/surfaceMatching.py, on the GPU.

  SurfaceMatchingParam(timeStep=.1, KparDiff=None, KparDist=None, sigmaKernel=6.5, sigmaDist=2.5,
                       sigmaError=1.0, errorType='measure', typeKernel='gauss')       surfaceMatching.py:19-50
  SurfaceMatching(Template, Target, ..., param, maxIter, regWeight, ..., testGradient=True, ...)
      .optimizeMatching()                                                          surfaceMatching.py:74-484

errorType selects the (fun_obj0, fun_obj, fun_objGrad) plug-in triple among
this library's surfaces.current/measure/varifold norms; a user-set triple is
honoured too (called with Surface objects).  Only affine='none' and
symmetric=False are provided.  VTK output of the iterates is not written.
Extra keywords: lineSearchPrecision ('fp64' default) -- the precision of the
data-term values compared by the line search (see registration_b200._matching);
cudaGraphs (True) -- replay each line-search trial (shot + data-term value)
from a captured CUDA graph instead of launching its kernels one by one.
"""
import logging

import numpy as np

from . import conjugateGradient as cg
from . import kernelFunctions as kfun
from . import surfaces
from ._matching import DeviceMatching, Direction  # noqa: F401


class SurfaceMatchingParam:
    def __init__(self, timeStep=.1, KparDiff=None, KparDist=None, sigmaKernel=6.5, sigmaDist=2.5, sigmaError=1.0,
                 errorType='measure', typeKernel='gauss'):
        self.timeStep = timeStep
        self.sigmaKernel = sigmaKernel
        self.sigmaDist = sigmaDist
        self.sigmaError = sigmaError
        self.typeKernel = typeKernel
        self.errorType = errorType
        if errorType in ('current', 'measure', 'varifold'):
            self.fun_obj0 = getattr(surfaces, errorType + 'Norm0')
            self.fun_obj = getattr(surfaces, errorType + 'NormDef')
            self.fun_objGrad = getattr(surfaces, errorType + 'NormGradient')
        else:
            logging.error('Unknown error Type: ' + self.errorType)
        self.KparDiff = KparDiff if KparDiff is not None else kfun.Kernel(name=self.typeKernel, sigma=sigmaKernel)
        self.KparDist = KparDist if KparDist is not None else kfun.Kernel(name='gauss', sigma=sigmaDist)


class SurfaceMatching(DeviceMatching):
    norm_module = surfaces
    tgt_vectors_attr = 'surfel'

    def __init__(self, Template=None, Target=None, fileTempl=None, fileTarg=None, param=None, maxIter=1000,
                 regWeight=1.0, affineWeight=1.0, verb=True, subsampleTargetSize=-1, rotWeight=None,
                 scaleWeight=None, transWeight=None, symmetric=False, testGradient=True, saveFile='evolution',
                 affine='none', outputDir='.', lineSearchPrecision='fp64', cudaGraphs=True):
        if Template is None:
            if fileTempl is None:
                raise ValueError('Please provide a template surface')
            Template = surfaces.Surface(filename=fileTempl)
        if Target is None:
            if fileTarg is None:
                raise ValueError('Please provide a target surface')
            Target = surfaces.Surface(filename=fileTarg)
        if subsampleTargetSize > 0:
            raise NotImplementedError('template simplification (VTK) is not provided')
        self.fv0 = surfaces.Surface(surf=Template)
        self.fv1 = surfaces.Surface(surf=Target)
        self.param = param if param is not None else SurfaceMatchingParam()
        self.saveRate = 10
        self.saveFile = saveFile
        self.outputDir = outputDir
        # surfaceMatching.py:126-129: orient the target like the template
        if self.fv0.surfVolume() * self.fv1.surfVolume() < 0:
            self.fv1.flipFaces()
        self.fvInit = surfaces.Surface(surf=self.fv0)
        self.fvDef = surfaces.Surface(surf=self.fvInit)
        self._init_state(maxIter, regWeight, verb, testGradient, affine, symmetric, lineSearchPrecision,
                         cudaGraphs=cudaGraphs)
        self.coeffAff1 = 1.
        self.coeffAff2 = 100.
        self.coeffAff = self.coeffAff1

    @staticmethod
    def shape_copy(s):
        return surfaces.Surface(surf=s)

    def optimizeMatching(self):
        """surfaceMatching.py:474-484: gradEps = max(1e-3, |g|/1e4), cg with epsInit 0.1."""
        grd = self.getGradient(self.gradCoeff)
        [grd2] = self.dotProduct(grd, [grd])
        self.gradEps = max(0.001, np.sqrt(grd2) / 10000)
        logging.info('Gradient lower bound: %f' % (self.gradEps))
        cg.cg(self, verb=self.verb, maxIter=self.maxIter, TestGradient=self.testGradient, epsInit=0.1)
