"""Python side of the ragged entry points (lddmm_ragged_* in include/lddmm_b200.h):
many independent point sets in ONE launch per kernel family, each segment with
its own size, kernel width and regularisation weight.

Used by the serving engine (many matching requests) and by template
estimation (one deformation per subject, surfaceTemplate.py:241-301).  Every
function takes device tensors in the concatenated layouts the C entry points
document and returns device tensors; nothing is read back to the host.
"""
import ctypes

import torch

from . import _lib
from .device import ptr, stream_handle, workspace

NORMS = {"current": 0, "measure": 1, "varifold": 2}


def i64(a):
    return (ctypes.c_int64 * len(a))(*[int(v) for v in a])


def f64(a):
    return (ctypes.c_double * len(a))(*[float(v) for v in a])


def kernel_order(K):
    """The f2py `ord` argument: > 4 selects the Gaussian (kernelFunctions.py:318-327)."""
    return 10 if K.name == "gauss" else int(K.order)


def offsets(counts):
    off = [0]
    for c in counts:
        off.append(off[-1] + int(c))
    return off


def shoot(x0, at, v_off, T, sigmas, order, regweights):
    """Euler shooting + deformation energy of every segment (lddmm_ragged_shoot_f32c).

    x0 (v_off[-1], d); at: segment s's (T, n_s, d) block at row T*v_off[s].
    Returns xt (segment s's (T+1, n_s, d) block at row (T+1)*v_off[s]) and
    energy (nseg,) = rw_s dt sum_t <a_t, K(x_t) a_t>."""
    nseg, d = len(v_off) - 1, x0.shape[1]
    x0, at = x0.contiguous(), at.contiguous()
    xt = torch.empty(((T + 1) * v_off[-1], d), dtype=torch.float64, device=x0.device)
    energy = torch.empty(nseg, dtype=torch.float64, device=x0.device)
    vo = i64(v_off)
    wsb = _lib.query("lddmm_ragged_shoot_f32c_workspace", nseg, vo, d, T, order)
    ws = workspace.get(wsb)
    _lib.call("lddmm_ragged_shoot_f32c", nseg, vo, d, ptr(x0), ptr(at), T, f64(sigmas), order, f64(regweights),
              ptr(xt), ptr(energy), ptr(ws), wsb, stream_handle())
    return xt, energy


def covector(xt, at, px1, v_off, T, sigmas, order, regweights):
    """Hamiltonian adjoint of every segment (lddmm_ragged_covector_f32c):
    pxt in xt's layout (pxt[T] = px1) and dat = 2 rw a_t - p_{t+1} in at's."""
    nseg, d = len(v_off) - 1, xt.shape[1]
    xt, at, px1 = xt.contiguous(), at.contiguous(), px1.contiguous()
    pxt = torch.empty_like(xt)
    dat = torch.empty_like(at)
    vo = i64(v_off)
    wsb = _lib.query("lddmm_ragged_covector_f32c_workspace", nseg, vo, d, T, order)
    ws = workspace.get(wsb)
    _lib.call("lddmm_ragged_covector_f32c", nseg, vo, d, ptr(xt), ptr(at), T, ptr(px1), f64(sigmas), order,
              f64(regweights), ptr(pxt), ptr(dat), ptr(ws), wsb, stream_handle())
    return pxt, dat


def applyk_segments(x, beta, starts, counts, sigmas, order):
    """Independent applyK segments with targets = sources = rows
    [starts[s], +counts[s]) of x and weights the same rows of beta
    (lddmm_ragged_applyk_f32c); the result is compact in segment order."""
    d, dimb = x.shape[1], beta.shape[1]
    x, beta = x.contiguous(), beta.contiguous()
    f = torch.empty((sum(int(c) for c in counts), dimb), dtype=torch.float64, device=x.device)
    st, cn = i64(starts), i64(counts)
    wsb = _lib.query("lddmm_ragged_applyk_f32c_workspace", len(starts), cn, cn, d, dimb, order)
    ws = workspace.get(wsb)
    _lib.call("lddmm_ragged_applyk_f32c", len(starts), st, cn, st, cn, d, ptr(x), ptr(x), ptr(beta), dimb,
              f64(sigmas), order, ptr(f), ptr(ws), wsb, stream_handle())
    return f


def dataterm(norm, verts, shapes, tcs, tvs, sigmas, order, precision, grad, frames=None):
    """Data terms of every segment (lddmm_ragged_dataterm_{f32c,f64}).

    verts: per-segment vertex tensors (n_s, d); shapes: their DeviceShape
    topologies; tcs / tvs: per-segment target centres and surfels / tangents,
    or None for the target self term Norm0 (cells against themselves);
    frames: None (per-segment bounding-box packing centres) or per-segment
    3-tuples of fixed centres.  Returns the energies (nseg,) or, with grad,
    the per-segment gradients w.r.t. the vertices."""
    k = shapes[0].cells.shape[1]
    d = verts[0].shape[1]
    dev = verts[0].device
    v_off, c_off, c2_off = [0], [0], [0]
    cells, vptr, vidx = [], [], []
    for v, shp, tc in zip(verts, shapes, tcs if tcs is not None else [None] * len(verts)):
        nc = shp.cells.shape[0]
        cells.append(shp.cells + v_off[-1])
        vptr.append(shp.vptr[:-1] + c_off[-1] * k)
        vidx.append(shp.vidx + c_off[-1] * k)
        v_off.append(v_off[-1] + v.shape[0])
        c_off.append(c_off[-1] + nc)
        c2_off.append(c2_off[-1] + (tc.shape[0] if tc is not None else 0))
    V = torch.cat(verts)
    C = torch.cat(cells)
    VP = torch.cat(vptr + [torch.full((1,), c_off[-1] * k, dtype=torch.int64, device=dev)])
    VI = torch.cat(vidx)
    C2 = torch.cat(list(tcs)) if tcs is not None else None
    S2 = torch.cat(list(tvs)) if tvs is not None else None
    nseg = len(verts)
    sfx = "f32c" if precision == "fp32c" else "f64"
    energy = None if grad else torch.empty(nseg, dtype=torch.float64, device=dev)
    px = torch.empty_like(V) if grad else None
    vo, co, c2o = i64(v_off), i64(c_off), i64(c2_off)
    wsb = _lib.query("lddmm_ragged_dataterm_%s_workspace" % sfx, nseg, k, NORMS[norm], vo, co, c2o, d, order,
                     0 if grad else 1, 1 if grad else 0)
    ws = workspace.get(wsb)
    _lib.call("lddmm_ragged_dataterm_" + sfx, nseg, k, NORMS[norm], vo, co, c2o, ptr(V), d, ptr(C),
              ptr(C2) if C2 is not None else None, ptr(S2) if S2 is not None else None,
              f64(sigmas), order, 1e-10, 1e-10,
              f64([c for fr in frames for c in fr]) if frames is not None else None,
              ptr(energy) if energy is not None else None, ptr(VP), ptr(VI),
              ptr(px) if px is not None else None, ptr(ws), wsb, stream_handle())
    if grad:
        return [px[v_off[i]:v_off[i + 1]] for i in range(nseg)]
    return energy
