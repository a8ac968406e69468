"""Triangulated surfaces and their data-attachment norms, with the names of
py-lddmm/surfaces.py, computed on the GPU.

  Surface(surf=None, filename=None, FV=None)     surfaces.py:24-75
    .vertices, .faces, .centers, .surfel, computeCentersAreas(), updateVertices(x),
    flipFaces(), surfVolume(), saveVTK(fileName)
  currentNorm0 / currentNormDef / currentNormGradient      surfaces.py:1009-1089
  measureNorm0 / measureNormDef / measureNormGradient      surfaces.py:1092-1182
  varifoldNorm0 / varifoldNormDef / varifoldNormGradient   surfaces.py:1184-1276
  (and currentNorm / measureNorm / varifoldNorm = Def + Norm0)

The norms take the same arguments as the reference (fvDef, fv1, KparDist) and
return a float (value) or an (nv, 3) float64 array (gradient; a CUDA tensor
when the surface holds device vertices).  None of them forms an F x F array.
Reading meshes from .byu/.off/.vtk/.obj files (VTK) is not part of this library.
"""
import os

import numpy as np
import torch

from . import _dataterm as _dt


class Surface:
    def __init__(self, surf=None, filename=None, FV=None):
        if surf is not None:
            self.vertices = _copy(surf.vertices)
            self.faces = np.copy(surf.faces)
            self._dshape = getattr(surf, "_dshape", None)
        elif FV is not None:
            self.vertices = _copy(FV[1])
            self.faces = np.int_(np.asarray(FV[0]))
            self._dshape = None
        elif filename is not None:
            raise NotImplementedError("mesh file readers are not part of this library; build Surface(FV=[faces, v])")
        else:
            self.vertices = np.empty(0)
            self.faces = np.empty(0, dtype=np.int64)
            self.centers = np.empty(0)
            self.surfel = np.empty(0)
            self._dshape = None
            return
        self.computeCentersAreas()

    def computeCentersAreas(self):
        """face centres and area-weighted normals (surfaces.py:61-66)"""
        self.centers, self.surfel = _dt.cell_geometry(self.vertices, self.faces)

    def updateVertices(self, x0):
        """(surfaces.py:69-75)"""
        self.vertices = _copy(x0)
        self.computeCentersAreas()

    def flipFaces(self):
        """(surfaces.py:261-263)"""
        self.faces = self.faces[:, [0, 2, 1]]
        self._dshape = None
        self.computeCentersAreas()

    def surfVolume(self):
        """sum over faces of det(v0, v1, v2)/6 (surfaces.py:711-717)"""
        v = _np(self.vertices)[self.faces]
        return float((np.linalg.det(v) / 6).sum())

    def device_shape(self):
        if self._dshape is None:
            self._dshape = _dt.DeviceShape(self.faces, len(self.vertices))
        return self._dshape

    def saveVTK(self, fileName, scalars=None, normals=None, scal_name='scalars'):
        """ASCII legacy VTK polydata (points and triangles, optional point scalars)."""
        V = _np(self.vertices)
        F = self.faces
        d = os.path.dirname(fileName)
        if d:
            os.makedirs(d, exist_ok=True)
        with open(fileName, 'w') as fh:
            fh.write('# vtk DataFile Version 3.0\nSurface Data\nASCII\nDATASET POLYDATA\n')
            fh.write('\nPOINTS {0:d} float'.format(V.shape[0]))
            for p in V:
                fh.write('\n{0: f} {1: f} {2: f}'.format(p[0], p[1], p[2]))
            fh.write('\nPOLYGONS {0:d} {1:d}'.format(F.shape[0], 4 * F.shape[0]))
            for f in F:
                fh.write('\n3 {0:d} {1:d} {2:d}'.format(f[0], f[1], f[2]))
            if scalars is not None:
                fh.write('\nPOINT_DATA {0:d}\nSCALARS {1} float 1\nLOOKUP_TABLE default'.format(V.shape[0], scal_name))
                for s in np.asarray(scalars):
                    fh.write('\n {0: .5f}'.format(s))
            fh.write('\n')


def _copy(x):
    if isinstance(x, torch.Tensor):
        return x.detach().clone()
    return np.array(x, dtype=np.float64, copy=True)


def _np(x):
    return x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


def _value(norm, fv, tgt, K, eps_def=1e-10, eps_tgt=1e-10):
    e, _ = _dt.dataterm(norm, fv.vertices, fv.device_shape(), None if tgt is None else tgt.centers,
                        None if tgt is None else tgt.surfel, K, energy=True, grad=False, eps1=eps_def, eps2=eps_tgt)
    return float(e)


def _gradient(norm, fvDef, fv1, K):
    _, px = _dt.dataterm(norm, fvDef.vertices, fvDef.device_shape(), fv1.centers, fv1.surfel, K, energy=False,
                         grad=True)
    return px if isinstance(fvDef.vertices, torch.Tensor) else px.cpu().numpy()


# --- current (surfaces.py:1008-1089) ----------------------------------------
def currentNorm0(fv1, KparDist):
    return _value("current", fv1, None, KparDist)


def currentNormDef(fvDef, fv1, KparDist):
    return _value("current", fvDef, fv1, KparDist)


def currentNorm(fvDef, fv1, KparDist):
    return currentNormDef(fvDef, fv1, KparDist) + currentNorm0(fv1, KparDist)


def currentNormGradient(fvDef, fv1, KparDist):
    return _gradient("current", fvDef, fv1, KparDist)


# --- measure (surfaces.py:1091-1182) ----------------------------------------
def measureNorm0(fv1, KparDist):
    return _value("measure", fv1, None, KparDist)


def measureNormDef(fvDef, fv1, KparDist):
    return _value("measure", fvDef, fv1, KparDist)


def measureNorm(fvDef, fv1, KparDist):
    return measureNormDef(fvDef, fv1, KparDist) + measureNorm0(fv1, KparDist)


def measureNormGradient(fvDef, fv1, KparDist):
    return _gradient("measure", fvDef, fv1, KparDist)


# --- varifold (surfaces.py:1184-1276) ---------------------------------------
def varifoldNorm0(fv1, KparDist):
    return _value("varifold", fv1, None, KparDist)


def varifoldNormDef(fvDef, fv1, KparDist):
    return _value("varifold", fvDef, fv1, KparDist)


def varifoldNorm(fvDef, fv1, KparDist):
    return varifoldNormDef(fvDef, fv1, KparDist) + varifoldNorm0(fv1, KparDist)


def varifoldNormGradient(fvDef, fv1, KparDist):
    return _gradient("varifold", fvDef, fv1, KparDist)
