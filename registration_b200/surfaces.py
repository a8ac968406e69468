"""Triangulated surfaces and their data-attachment norms, with the names of
py-lddmm/surfaces.py, computed on the GPU.

  Surface(surf=None, filename=None, FV=None)     surfaces.py:24-75
    .vertices, .faces, .centers, .surfel, computeCentersAreas(), updateVertices(x),
    flipFaces(), surfVolume(), readbyu / readOFF / readVTK / readOBJ, savebyu, saveVTK / saveVTK2,
    computeVertexArea(), computeVertexNormals()                               surfaces.py:77-139, 711-985
  readMultipleByu, saveEvolution, vtkFields, readskip                          surfaces.py:16-21, 988-1005, 1279
  currentNorm0 / currentNormDef / currentNormGradient      surfaces.py:1009-1089
  measureNorm0 / measureNormDef / measureNormGradient      surfaces.py:1092-1182
  varifoldNorm0 / varifoldNormDef / varifoldNormGradient   surfaces.py:1184-1276
  (and currentNorm / measureNorm / varifoldNorm = Def + Norm0)

The norms take the same arguments as the reference (fvDef, fv1, KparDist) and
return a float (value) or an (nv, 3) float64 array (gradient; a CUDA tensor
when the surface holds device vertices).  None of them forms an F x F array.
Mesh files (.byu / .off / legacy ASCII .vtk / .obj), vertex areas and vertex
normals: registration_b200.meshio (host side).
"""
import glob
import logging
import os

import numpy as np
import torch

from . import _dataterm as _dt
from . import meshio


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
            self._dshape = None
            ext = os.path.splitext(filename)[1]
            readers = {'.byu': self.readbyu, '.off': self.readOFF, '.vtk': self.readVTK, '.obj': self.readOBJ}
            if ext not in readers:
                logging.error('Unknown Surface Extension: %s', ext)
                self.vertices = np.empty(0)
                self.faces = np.empty(0, dtype=np.int64)
                self.centers = np.empty(0)
                self.surfel = np.empty(0)
                return
            readers[ext](filename)
            return
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
        self._centers, self._surfel = _dt.cell_geometry(self.vertices, self.faces)
        self._stale = False

    def updateVertices(self, x0):
        """(surfaces.py:69-75); the centres and normals follow on first use."""
        self.vertices = _copy(x0)
        self._stale = True

    # centres / surfel of the current vertices, recomputed after updateVertices when read
    @property
    def centers(self):
        if getattr(self, "_stale", False):
            self.computeCentersAreas()
        return self._centers

    @centers.setter
    def centers(self, c):
        self._centers = c

    @property
    def surfel(self):
        if getattr(self, "_stale", False):
            self.computeCentersAreas()
        return self._surfel

    @surfel.setter
    def surfel(self, s):
        self._surfel = s

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

    def _set_mesh(self, vertices, faces):
        self.vertices = vertices
        self.faces = np.int_(faces)
        self._dshape = None
        self.computeCentersAreas()

    # -- files (surfaces.py:719-985) -------------------------------------------------------
    def readbyu(self, byufile):
        """(surfaces.py:757-805)"""
        self._set_mesh(*meshio.read_byu(byufile))

    def readOFF(self, offfile):
        """(surfaces.py:719-754)"""
        self._set_mesh(*meshio.read_off(offfile))

    def readVTK(self, fileName):
        """legacy ASCII POLYDATA (the reference reads it through VTK, surfaces.py:928-955)"""
        self._set_mesh(*meshio.read_vtk(fileName))

    def readOBJ(self, fileName):
        """(the reference reads it through VTK, surfaces.py:957-985)"""
        self._set_mesh(*meshio.read_obj(fileName))

    def savebyu(self, byufile):
        """(surfaces.py:807-849)"""
        meshio.write_byu(byufile, _np(self.vertices), self.faces)

    def saveVTK(self, fileName, scalars=None, normals=None, tensors=None, scal_name='scalars', vectors=None,
                vect_name='vectors'):
        """(surfaces.py:851-867)"""
        vf = meshio.vtkFields()
        if scalars is not None:
            vf.scalars += [scal_name, _np(scalars)]
        if vectors is not None:
            vf.vectors += [vect_name, _np(vectors)]
        if normals is not None:
            vf.normals += ['normals', _np(normals)]
        if tensors is not None:
            vf.tensors += ['tensors', _np(tensors)]
        self.saveVTK2(fileName, vf)

    def saveVTK2(self, fileName, vtkFields=None):
        """(surfaces.py:869-925)"""
        d = os.path.dirname(fileName)
        if d:
            os.makedirs(d, exist_ok=True)
        meshio.write_vtk(fileName, _np(self.vertices), self.faces, vtkFields)

    # -- per-vertex geometry (surfaces.py:77-139) ------------------------------------------------
    def computeVertexArea(self):
        """(AV (nv, 1), AF (nf, 1)) (surfaces.py:77-126)"""
        return meshio.vertex_area(_np(self.vertices), self.faces)

    def computeVertexNormals(self):
        """(surfaces.py:128-139)"""
        self.computeCentersAreas()
        return meshio.vertex_normals(_np(self.vertices), self.faces)


def readMultipleByu(regexp, Nmax=0):
    """Surfaces of the .byu files matching a glob pattern (surfaces.py:988-997)."""
    files = glob.glob(regexp)
    nm = min(Nmax, len(files)) if Nmax > 0 else len(files)
    return [Surface(filename=files[k]) for k in range(nm)]


def saveEvolution(fileName, fv0, xt):
    """One .byu file per time step of a trajectory xt (T+1, N, 3) (surfaces.py:1000-1005)."""
    fv = Surface(surf=fv0)
    xt = _np(xt)
    for k in range(xt.shape[0]):
        meshio.write_byu(fileName + '{0: 02d}'.format(k) + '.byu', xt[k], fv.faces)


vtkFields = meshio.vtkFields
readskip = meshio.readskip


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
