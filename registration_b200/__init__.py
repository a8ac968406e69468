"""B200 (sm_100a) implementation of the py-lddmm point-LDDMM hot path.

Modules mirror the reference's module names and call signatures:
  kernelFunctions   Kernel / KernelSpec (applyK, applyDiffKT, applyDivergence)
  pointEvolution    landmarkDirectEvolutionEuler, landmarkEPDiff,
                    landmarkHamiltonianCovector, landmarkHamiltonianGradient
  surfaces, curves  Surface / Curve and the current / measure / varifold norms
  surfaceMatching, curveMatching, matchingParam, conjugateGradient, gradientDescent
  surfaceTemplate   SurfaceTemplate (template estimation over many subjects)
  serving           ServingEngine (continuous batching of matching requests)
The arithmetic runs in liblddmm_b200.so (C ABI: include/lddmm_b200.h), built
with `python -m registration_b200.build`; there is no CPU fallback.
"""
__all__ = ["kernelFunctions", "pointEvolution", "surfaces", "curves", "surfaceMatching", "curveMatching",
           "matchingParam", "conjugateGradient", "gradientDescent", "geometry", "surfaceTemplate", "serving"]
