"""MatchingParam (py-lddmm/matchingParam.py:10-25): time step, kernels and error
normalisation shared by the matching problems."""
from . import kernelFunctions as kfun


class MatchingParam:
    def __init__(self, timeStep=.1, KparDiff=None, KparDist=None, sigmaKernel=6.5, sigmaDist=2.5, sigmaError=1.0,
                 errorType='measure', typeKernel='gauss'):
        self.timeStep = timeStep
        self.sigmaKernel = sigmaKernel
        self.sigmaDist = sigmaDist
        self.sigmaError = sigmaError
        self.typeKernel = typeKernel
        self.errorType = errorType
        self.KparDiff = KparDiff if KparDiff is not None else kfun.Kernel(name=self.typeKernel, sigma=sigmaKernel)
        self.KparDist = KparDist if KparDist is not None else kfun.Kernel(name='gauss', sigma=sigmaDist)
