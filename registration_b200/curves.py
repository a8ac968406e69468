"""Polygonal curves and their data-attachment norms, with the names of
py-lddmm/curves.py, computed on the GPU.

  Curve(curve=None, filename=None, FV=None, pointSet=None, isOpen=False)  curves.py:15-75
    .vertices, .faces (edges), .centers, .lenel, computeCentersLengths(), updateVertices(x)
  currentNorm0 / currentNormDef / currentNormGradient   curves.py:539-613
  measureNorm0 / measureNormDef / measureNormGradient   curves.py:621-703
  (no varifold for curves, as in the reference)

curves.measureNorm0 keeps the reference's missing 1e-10 under the square root
(curves.py:624); the other measure weights use sqrt(|t|^2 + 1e-10).  An open
curve built from a point set keeps the reference's zero-length last edge.
"""
import numpy as np
import torch

from . import _dataterm as _dt
from .surfaces import _copy, _np


class Curve:
    def __init__(self, curve=None, filename=None, FV=None, pointSet=None, isOpen=False):
        self._dshape = None
        if curve is not None:
            self.vertices = _copy(curve.vertices)
            self.faces = np.copy(curve.faces)
            self._dshape = getattr(curve, "_dshape", None)
        elif FV is not None:
            self.vertices = _copy(FV[1])
            self.faces = np.int_(np.asarray(FV[0]))
        elif pointSet is not None:
            self.vertices = _copy(pointSet)
            n = len(self.vertices)
            self.faces = np.stack([np.arange(n), np.arange(1, n + 1)], axis=1).astype(np.int64)
            # closed: last edge (n-1, 0); open: the reference leaves the last
            # row at (0, 0), a zero-length edge (curves.py:27-31) -- kept.
            self.faces[-1] = (n - 1, 0) if not isOpen else (0, 0)
        elif filename is not None:
            raise NotImplementedError("curve file readers are not part of this library")
        else:
            self.vertices = np.empty(0)
            self.faces = np.empty(0, dtype=np.int64)
            self.centers = np.empty(0)
            self.lenel = np.empty(0)
            return
        self.computeCentersLengths()

    def computeCentersLengths(self):
        """edge centres and tangent vectors (curves.py:58-64)"""
        self._centers, self._lenel = _dt.cell_geometry(self.vertices, self.faces)
        self._stale = False

    def updateVertices(self, x0):
        """The centres and tangents follow on first use."""
        self.vertices = _copy(x0)
        self._stale = True

    @property
    def centers(self):
        if getattr(self, "_stale", False):
            self.computeCentersLengths()
        return self._centers

    @centers.setter
    def centers(self, c):
        self._centers = c

    @property
    def lenel(self):
        if getattr(self, "_stale", False):
            self.computeCentersLengths()
        return self._lenel

    @lenel.setter
    def lenel(self, v):
        self._lenel = v

    def device_shape(self):
        if self._dshape is None:
            self._dshape = _dt.DeviceShape(self.faces, len(self.vertices))
        return self._dshape


def _value(norm, fv, tgt, K, eps_def=1e-10, eps_tgt=1e-10):
    e, _ = _dt.dataterm(norm, fv.vertices, fv.device_shape(), None if tgt is None else tgt.centers,
                        None if tgt is None else tgt.lenel, K, energy=True, grad=False, eps1=eps_def, eps2=eps_tgt)
    return float(e)


def _gradient(norm, fvDef, fv1, K):
    _, px = _dt.dataterm(norm, fvDef.vertices, fvDef.device_shape(), fv1.centers, fv1.lenel, K, energy=False,
                         grad=True)
    return px if isinstance(fvDef.vertices, torch.Tensor) else px.cpu().numpy()


def currentNorm0(fv1, KparDist):
    return _value("current", fv1, None, KparDist)


def currentNormDef(fvDef, fv1, KparDist):
    return _value("current", fvDef, fv1, KparDist)


def currentNorm(fvDef, fv1, KparDist):
    return currentNormDef(fvDef, fv1, KparDist) + currentNorm0(fv1, KparDist)


def currentNormGradient(fvDef, fv1, KparDist):
    return _gradient("current", fvDef, fv1, KparDist)


def measureNorm0(fv1, KparDist):
    return _value("measure", fv1, None, KparDist, eps_def=0.0)


def measureNormDef(fvDef, fv1, KparDist):
    return _value("measure", fvDef, fv1, KparDist)


def measureNorm(fvDef, fv1, KparDist):
    return measureNormDef(fvDef, fv1, KparDist) + measureNorm0(fv1, KparDist)


def measureNormGradient(fvDef, fv1, KparDist):
    return _gradient("measure", fvDef, fv1, KparDist)
