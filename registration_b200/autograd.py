"""The matching objective as a torch.autograd.Function with a hand-written backward.

    E(a, x0) = sum_t rw dt <a_t, K(x_t) a_t>  +  D(x_T) / sigmaError^2
    x_{t+1}  = x_t + dt K(x_t) a_t,   dt = 1/T

(objectiveFunDef + dataTerm of py-lddmm/surfaceMatching.py:187-221, 181-185).
The backward is the discrete Hamiltonian adjoint of the Euler scheme
(pointEvolution.py:735-817): p_T = -grad D(x_T) / sigmaError^2,
p_t = p_{t+1} + dt grad_x H(x_t, p_{t+1}, a_t), and

    dE/da_t = dt K(x_t) (2 rw a_t - p_{t+1})     (the reference's dat_t, mapped
                                                  from the K-metric to the
                                                  Euclidean gradient)
    dE/dx0  = -p_0.

Trajectory checkpointing: with ``checkpoint_every = c`` the forward keeps only
x_0, x_c, x_2c, ... and x_T; the backward re-shoots each segment from its
checkpoint (same kernels, same dt: bit-identical states) and runs the adjoint
over it.  ``checkpoint_every=None`` stores the whole trajectory unless
(T+1) N dim doubles exceed ``memory_budget_bytes``, in which case segments of
sqrt(T) steps are used.
"""
import math

import torch

from . import _dataterm as _dt
from . import pointEvolution as evol
from .device import require_cuda


class Geometry:
    """Fixed pieces of a matching problem: template topology, target cells, kernels."""

    def __init__(self, template, target, KparDiff, KparDist, errorType, sigmaError=1.0, regweight=1.0,
                 vectors_attr=None):
        require_cuda()
        self.dshape = template.device_shape()
        attr = vectors_attr or ('surfel' if hasattr(target, 'surfel') else 'lenel')
        self.tc = torch.as_tensor(target.centers, dtype=torch.float64).cuda()
        self.tv = torch.as_tensor(getattr(target, attr), dtype=torch.float64).cuda()
        self.KparDiff = KparDiff
        self.KparDist = KparDist
        self.errorType = errorType
        self.sigmaError = sigmaError
        self.regweight = regweight

    def data(self, x, energy=True, grad=False):
        e, px = _dt.dataterm(self.errorType, x, self.dshape, self.tc, self.tv, self.KparDist, energy=energy,
                             grad=grad)
        s = 1.0 / self.sigmaError ** 2
        return (e * s if e is not None else None), (px * s if px is not None else None)


def _segments(T, c):
    return [(s, min(s + c, T)) for s in range(0, T, c)]


class LDDMMObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, at, x0, geom, checkpoint_every, memory_budget_bytes):
        T, n, d = at.shape
        dt = 1.0 / T
        if checkpoint_every is None:
            full = (T + 1) * n * d * 8
            checkpoint_every = T if full <= memory_budget_bytes else max(1, int(math.sqrt(T)))
        c = int(checkpoint_every)
        K = geom.KparDiff
        reg = torch.zeros((), dtype=torch.float64, device=at.device)
        x = x0
        checkpoints = {}
        xt_full = None
        for (s, e) in _segments(T, c):
            xt_seg, en = evol.shoot(x, at[s:e], K, regweight=geom.regweight, with_energy=True, dt=dt)
            reg = reg + en
            if c >= T:
                xt_full = xt_seg
            else:
                checkpoints[s] = x.clone() if s == 0 else x
            x = xt_seg[-1].clone()
        data, _ = geom.data(x, energy=True)
        ctx.geom = geom
        ctx.c = c
        ctx.checkpoints = checkpoints
        ctx.xt_full = xt_full
        ctx.save_for_backward(at, x0, x)
        return reg + data

    @staticmethod
    def backward(ctx, gE):
        at, x0, xT = ctx.saved_tensors
        geom = ctx.geom
        K = geom.KparDiff
        T = at.shape[0]
        dt = 1.0 / T
        _, pxT = geom.data(xT, energy=False, grad=True)
        p = -pxT
        grad_at = torch.empty_like(at)
        for (s, e) in reversed(_segments(T, ctx.c)):
            if ctx.xt_full is not None:
                xt_seg = ctx.xt_full[s:e + 1]
            else:
                xt_seg, _ = evol.shoot(ctx.checkpoints[s], at[s:e], K, dt=dt)
            pxt_seg, dat_seg = evol.covector(xt_seg, at[s:e], p, K, geom.regweight, with_dat=True, dt=dt)
            for t in range(e - s):
                grad_at[s + t] = dt * K.applyK(xt_seg[t], dat_seg[t])
            p = pxt_seg[0]
        g = gE.to(torch.float64)
        return g * grad_at, g * (-p), None, None, None


def lddmm_objective(at, x0, geom, checkpoint_every=None, memory_budget_bytes=8 << 30):
    """E(a, x0) as a differentiable torch scalar (FP64), see the module docstring."""
    return LDDMMObjective.apply(at, x0, geom, checkpoint_every, memory_budget_bytes)
