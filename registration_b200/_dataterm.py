"""Shared host code of the surface / curve data-attachment terms.

Calls lddmm_dataterm_* (include/lddmm_b200.h) with the deformed shape's
vertices and cells and the target shape's centres and surfels/tangents.
"""
import numpy as np
import torch

from . import _lib
from .device import ptr, require_cuda, stream_handle, to_dev, workspace
from .kernelFunctions import _suffix

NORMS = {"current": 0, "measure": 1, "varifold": 2}


def vertex_csr(cells, nv):
    """Vertex -> (cell, corner) incidence, entries cell*k + corner, ordered per
    vertex by corner then cell (the accumulation order of the reference's
    three per-corner loops, surfaces.py:1074-1087)."""
    cells = np.asarray(cells, dtype=np.int64)
    nc, k = cells.shape
    vert = cells.reshape(-1)
    codes = np.arange(nc * k, dtype=np.int64)
    order = np.lexsort((codes // k, codes % k, vert))
    counts = np.bincount(vert, minlength=nv)
    ptr_ = np.zeros(nv + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr_[1:])
    return ptr_, codes[order]


class DeviceShape:
    """Device copies of a shape's topology (cells, CSR) -- built once."""

    def __init__(self, cells, nv):
        cells = np.ascontiguousarray(np.asarray(cells, dtype=np.int64))
        if cells.size and (cells.min() < 0 or cells.max() >= nv):
            raise ValueError("cell indices out of range")
        self.cells_np = cells
        self.nv = nv
        p, i = vertex_csr(cells, nv)
        self.cells = torch.from_numpy(cells).cuda()
        self.vptr = torch.from_numpy(p).cuda()
        self.vidx = torch.from_numpy(i).cuda()


def cell_geometry(vertices, cells):
    """Centres and surfels (triangles) or tangents (edges), as in the reference."""
    v = vertices
    if isinstance(v, torch.Tensor):
        c = torch.as_tensor(cells, device=v.device)
        x = [v[c[:, j]] for j in range(c.shape[1])]
        if c.shape[1] == 3:
            return (x[0] + x[1] + x[2]) / 3, torch.linalg.cross(x[1] - x[0], x[2] - x[0])
        return (x[0] + x[1]) / 2, x[1] - x[0]
    x = [v[cells[:, j]] for j in range(cells.shape[1])]
    if cells.shape[1] == 3:
        return (x[0] + x[1] + x[2]) / 3, np.cross(x[1] - x[0], x[2] - x[0])
    return (x[0] + x[1]) / 2, x[1] - x[0]


def dataterm(norm, vertices, dshape, tgt_centers, tgt_vectors, K, energy=True, grad=False, eps1=1e-10, eps2=1e-10,
             energy_out=None):
    """Returns (energy 0-d tensor or None, px tensor or None), on the device.

    vertices: (nv, d) of the deformed shape S1 with topology `dshape`;
    tgt_centers / tgt_vectors: (nc2, d) of S2 (None for Norm0 of S1);
    energy_out: a 0-d FP64 device tensor that receives the energy."""
    require_cuda()
    if K.name == 'none':
        raise ValueError("a kernel is required")
    v = to_dev(vertices)
    nv, d = v.shape
    k = dshape.cells.shape[1]
    nc = dshape.cells.shape[0]
    if tgt_centers is None:
        c2 = s2 = None
        nc2 = 0
    else:
        c2, s2 = to_dev(tgt_centers), to_dev(tgt_vectors)
        nc2 = c2.shape[0]
    sfx = _suffix(K.precision)
    if energy and energy_out is not None:
        e = energy_out
    else:
        e = torch.empty((), dtype=torch.float64, device=v.device) if energy else None
    px = torch.empty((nv, d), dtype=torch.float64, device=v.device) if grad else None
    wsb = _lib.query("lddmm_dataterm_%s_workspace" % sfx, k, NORMS[norm], nv, d, nc, nc2, int(K.order),
                     1 if energy else 0, 1 if grad else 0)
    ws = workspace.get(wsb)
    _lib.call("lddmm_dataterm_" + sfx, k, NORMS[norm], ptr(v), nv, d, ptr(dshape.cells), nc,
              ptr(c2) if c2 is not None else None, ptr(s2) if s2 is not None else None, nc2, float(K.sigma),
              int(K.order), float(eps1), float(eps2), ptr(e) if e is not None else None, ptr(dshape.vptr),
              ptr(dshape.vidx), ptr(px) if px is not None else None, ptr(ws), wsb, stream_handle())
    return e, px


def value_batch(norm, vertices, dshape, tgt_centers, tgt_vectors, K, eps1=1e-10, eps2=1e-10, energy_out=None):
    """Values (nbatch,) of the vertex sets vertices[b] of one topology `dshape`
    against one target: vertices is an (nbatch, nv, d) FP64 device view whose
    vertex sets are contiguous (any stride between them, e.g. xt[:, -1] of
    batched trajectories); energy_out: a contiguous (nbatch,) FP64 device tensor.
    energy[b] is bit-identical to dataterm(norm, vertices[b], ...)."""
    require_cuda()
    if K.name == 'none':
        raise ValueError("a kernel is required")
    v = vertices
    if not (isinstance(v, torch.Tensor) and v.is_cuda and v.dtype == torch.float64 and v.dim() == 3):
        raise ValueError("vertices must be an (nbatch, nv, d) FP64 device tensor")
    B, nv, d = v.shape
    if v.stride(2) != 1 or v.stride(1) != d or (B > 1 and v.stride(0) < nv * d):
        raise ValueError("each vertex set must be contiguous and the sets must not overlap")
    k = dshape.cells.shape[1]
    nc = dshape.cells.shape[0]
    if tgt_centers is None:
        c2 = s2 = None
        nc2 = 0
    else:
        c2, s2 = to_dev(tgt_centers), to_dev(tgt_vectors)
        nc2 = c2.shape[0]
    sfx = _suffix(K.precision)
    e = energy_out if energy_out is not None else torch.empty(B, dtype=torch.float64, device=v.device)
    if tuple(e.shape) != (B,) or not e.is_contiguous():
        raise ValueError("energy_out must be a contiguous (nbatch,) tensor")
    wsb = _lib.query("lddmm_dataterm_value_batch_%s_workspace" % sfx, k, NORMS[norm], nv, d, nc, nc2, int(K.order), B)
    ws = workspace.get(wsb)
    _lib.call("lddmm_dataterm_value_batch_" + sfx, k, NORMS[norm], ptr(v), nv, d, ptr(dshape.cells), nc,
              ptr(c2) if c2 is not None else None, ptr(s2) if s2 is not None else None, nc2, float(K.sigma),
              int(K.order), float(eps1), float(eps2), B, v.stride(0) if B > 1 else nv * d, ptr(e), ptr(ws), wsb,
              stream_handle())
    return e
