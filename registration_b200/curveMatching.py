"""Curve matching with the interface of py-lddmm/curveMatching.py, on the GPU.

  CurveMatchingParam(timeStep=.1, KparDiff=None, KparDist=None, sigmaKernel=6.5, sigmaDist=2.5,
                     sigmaError=1.0, errorType='measure', typeKernel='gauss')        curveMatching.py:19-35
  CurveMatching(Template, Target, ..., param, maxIter, regWeight, ..., gradLB=0.001, saveRate=10,
                testGradient=False, ...).optimizeMatching()                         curveMatching.py:58-352

optimizeMatching runs conjugateGradient.cg with its default epsInit = 10, as the
reference does; gradEps = max(gradLB, |g|/1e4).  Only affine='none'.
"""
import logging

import numpy as np

from . import conjugateGradient as cg
from . import curves
from . import gradientDescent
from . import kernelFunctions as kfun
from ._matching import DeviceMatching, Direction  # noqa: F401
from .matchingParam import MatchingParam


class CurveMatchingParam(MatchingParam):
    def __init__(self, timeStep=.1, KparDiff=None, KparDist=None, sigmaKernel=6.5, sigmaDist=2.5, sigmaError=1.0,
                 errorType='measure', typeKernel='gauss'):
        MatchingParam.__init__(self, timeStep=timeStep, KparDiff=KparDiff, KparDist=KparDist,
                               sigmaKernel=sigmaKernel, sigmaDist=sigmaDist, sigmaError=sigmaError,
                               errorType=errorType, typeKernel=typeKernel)
        if errorType in ('current', 'measure'):
            self.fun_obj0 = getattr(curves, errorType + 'Norm0')
            self.fun_obj = getattr(curves, errorType + 'NormDef')
            self.fun_objGrad = getattr(curves, errorType + 'NormGradient')
        else:
            logging.error('Unknown error Type: %s' % errorType)


class CurveMatching(DeviceMatching):
    norm_module = curves
    tgt_vectors_attr = 'lenel'

    def __init__(self, Template=None, Target=None, fileTempl=None, fileTarg=None, param=None, maxIter=1000,
                 regWeight=1.0, affineWeight=1.0, verb=True, gradLB=0.001, saveRate=10, rotWeight=None,
                 scaleWeight=None, transWeight=None, testGradient=False, saveFile='evolution', affine='none',
                 outputDir='.', lineSearchPrecision='fp64', cudaGraphs=True):
        if Template is None or Target is None:
            raise ValueError('Please provide template and target curves (file readers are not provided)')
        self.fv0 = curves.Curve(curve=Template)
        self.fv1 = curves.Curve(curve=Target)
        self.param = param if param is not None else CurveMatchingParam()
        self.fvDef = curves.Curve(curve=self.fv0)
        self.gradLB = gradLB
        self.saveRate = saveRate
        self.saveFile = saveFile
        self.outputDir = outputDir
        self._init_state(maxIter, regWeight, verb, testGradient, affine, False, lineSearchPrecision,
                         cudaGraphs=cudaGraphs)

    @staticmethod
    def shape_copy(c):
        return curves.Curve(curve=c)

    def optimizeMatching(self, optimizer='cg'):
        """curveMatching.py:342-352."""
        grd = self.getGradient(self.gradCoeff)
        [grd2] = self.dotProduct(grd, [grd])
        self.gradEps = max(self.gradLB, np.sqrt(grd2) / 10000)
        logging.info('Gradient bound: %f' % self.gradEps)
        if optimizer == 'cg':
            cg.cg(self, verb=self.verb, maxIter=self.maxIter, TestGradient=self.testGradient)
        else:
            gradientDescent.descend(self, verb=self.verb, maxIter=self.maxIter)
