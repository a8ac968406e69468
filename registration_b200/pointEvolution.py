"""Landmark evolution with the signatures of py-lddmm/pointEvolution.py, on the GPU.

  landmarkDirectEvolutionEuler (pointEvolution.py:666-730)
  landmarkEPDiff               (pointEvolution.py:599-658)
  landmarkHamiltonianCovector  (pointEvolution.py:735-765)
  landmarkHamiltonianGradient  (pointEvolution.py:793-817)
  secondOrderEvolution / Hamiltonian / Covector / Gradient (pointEvolution.py:882-1091)

The plain shot and the adjoint each run as one fused C-ABI call (one kernel
sweep + one combine per time step).  The optional outputs of the direct
evolution (withPointSet / withJacobian / withNormals) are evaluated step by
step with the kernel-sum operators.  Affine parts: only the all-zero affine
arguments that the matching code passes for affine='none' are accepted.

numpy in -> numpy out; CUDA tensors in -> CUDA tensors out.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .device import is_device, output_like, ptr, require_cuda, stream_handle, to_dev, workspace
from .kernelFunctions import _suffix


def _check_affine(affine):
    if affine is None:
        return
    for part in affine:
        arr = part.detach().cpu().numpy() if isinstance(part, torch.Tensor) else np.asarray(part)
        if arr.size and np.any(arr != 0):
            raise NotImplementedError("non-zero affine components are not supported (affine='none' only)")


def _kernel_args(K):
    if K.name == 'none':
        raise ValueError("a kernel is required")
    return float(K.sigma), int(K.order), _suffix(K.precision)


def shoot(x0, at, KparDiff, regweight=1.0, with_energy=False, dt=None, energy_out=None):
    """Device call: returns (xt, energy) with energy = sum_t rw dt <a_t, K(x_t) a_t> (a 0-d tensor) or None.
    dt defaults to 1/T; pass it to shoot a segment of a longer trajectory.  energy_out: a 0-d FP64
    device tensor (e.g. a view into a larger buffer) that receives the energy."""
    require_cuda()
    x0d = to_dev(x0)
    atd = to_dev(at)
    T, n, d = atd.shape
    if x0d.shape != (n, d):
        raise ValueError("x0 must be (N, dim) and at (T, N, dim)")
    sigma, order, sfx = _kernel_args(KparDiff)
    xt = torch.empty((T + 1, n, d), dtype=torch.float64, device=x0d.device)
    if energy_out is not None:
        energy = energy_out
    else:
        energy = torch.empty((), dtype=torch.float64, device=x0d.device) if with_energy else None
    wsb = _lib.query("lddmm_shoot_%s_workspace" % sfx, n, d, T)
    ws = workspace.get(wsb)
    _lib.call("lddmm_shoot_" + sfx, ptr(x0d), n, d, ptr(atd), T, float(dt or 0.0), sigma, order, float(regweight), ptr(xt),
              ptr(energy) if energy is not None else None, ptr(ws), wsb, stream_handle())
    return xt, energy


def shoot_along(x0, at, dir_, eps, KparDiff, regweight=1.0, at_try=None, energy_out=None):
    """Device call: the shot of the trial momenta at - eps dir (eps a 0-d FP64 device
    tensor), written to at_try (allocated if None); returns (at_try, xt, energy)."""
    require_cuda()
    x0d, atd, dd = to_dev(x0), to_dev(at), to_dev(dir_)
    T, n, d = atd.shape
    if dd.shape != atd.shape or x0d.shape != (n, d):
        raise ValueError("x0 must be (N, dim), at and dir (T, N, dim)")
    sigma, order, sfx = _kernel_args(KparDiff)
    if at_try is None:
        at_try = torch.empty_like(atd)
    xt = torch.empty((T + 1, n, d), dtype=torch.float64, device=x0d.device)
    energy = energy_out if energy_out is not None else torch.empty((), dtype=torch.float64, device=x0d.device)
    wsb = _lib.query("lddmm_shoot_%s_workspace" % sfx, n, d, T)
    ws = workspace.get(wsb)
    _lib.call("lddmm_shoot_along_" + sfx, ptr(x0d), n, d, ptr(atd), ptr(dd.contiguous()), ptr(eps), T, 0.0, sigma,
              order, float(regweight), ptr(at_try), ptr(xt), ptr(energy), ptr(ws), wsb, stream_handle())
    return at_try, xt, energy


def shoot_along_batch(x0, at, dir_, eps, KparDiff, regweight=1.0, at_try=None, xt=None, energy=None):
    """Device call: the shots of at - eps[b] dir for every step size of the FP64
    device vector eps (nbatch,); returns (at_try (nbatch, T, N, dim), xt
    (nbatch, T+1, N, dim), energy (nbatch,)), slot b bit-identical to
    shoot_along with eps[b].  Outputs given as arguments must be contiguous."""
    require_cuda()
    x0d, atd, dd = to_dev(x0), to_dev(at), to_dev(dir_)
    T, n, d = atd.shape
    if dd.shape != atd.shape or x0d.shape != (n, d):
        raise ValueError("x0 must be (N, dim), at and dir (T, N, dim)")
    if not (isinstance(eps, torch.Tensor) and eps.is_cuda and eps.dtype == torch.float64 and eps.dim() == 1
            and eps.is_contiguous() and eps.numel() >= 1):
        raise ValueError("eps must be a contiguous FP64 device vector of the step sizes")
    B = eps.numel()
    sigma, order, sfx = _kernel_args(KparDiff)
    want = {"at_try": (B, T, n, d), "xt": (B, T + 1, n, d), "energy": (B,)}
    outs = {"at_try": at_try, "xt": xt, "energy": energy}
    for k, shape in want.items():
        if outs[k] is None:
            outs[k] = torch.empty(shape, dtype=torch.float64, device=x0d.device)
        elif tuple(outs[k].shape) != shape or not outs[k].is_contiguous() or outs[k].dtype != torch.float64:
            raise ValueError("%s must be a contiguous FP64 tensor of shape %s" % (k, shape))
    wsb = _lib.query("lddmm_shoot_along_batch_%s_workspace" % sfx, n, d, T, B)
    ws = workspace.get(wsb)
    _lib.call("lddmm_shoot_along_batch_" + sfx, ptr(x0d), n, d, ptr(atd), ptr(dd), ptr(eps), B, T, 0.0, sigma,
              order, float(regweight), ptr(outs["at_try"]), ptr(outs["xt"]), ptr(outs["energy"]), ptr(ws), wsb,
              stream_handle())
    return outs["at_try"], outs["xt"], outs["energy"]


def trial_batch_size(n, d, ncells, ncells_target, shot_precision="fp32c", value_precision="fp64"):
    """Step sizes that one batched trial launch evaluates side by side (1: the
    problem is too large for the single-cluster kernels, batches would run one
    step size after the other)."""
    return max(1, _lib.query("lddmm_trial_batch_size", int(n), int(d), int(ncells), int(ncells_target),
                             int(shot_precision == "fp64"), int(value_precision == "fp64")))


def metric_dots(xt, g1, g2s, KparDiff):
    """Device call: the FP64 device vector (len(g2s),) of
    sum_t sum_k <g2[t][k], sum_j K(xt[t][k], xt[t][j]) g1[t][j]> over the T = len(g1)
    steps of the trajectory xt (T+1 or T, N, dim), one entry per g2 in g2s (<= 8);
    the metric inner products of Matching.dotProduct in two launches."""
    require_cuda()
    xtd, g1d = to_dev(xt), to_dev(g1)
    g2d = [to_dev(g) for g in g2s]
    T, n, d = g1d.shape
    if xtd.shape[0] < T or tuple(xtd.shape[1:]) != (n, d) or any(tuple(g.shape) != (T, n, d) for g in g2d):
        raise ValueError("xt must be (>= T, N, dim), g1 and every g2 (T, N, dim)")
    if not 1 <= len(g2d) <= 8:
        raise ValueError("1 to 8 directions g2")
    sigma, order, sfx = _kernel_args(KparDiff)
    out = torch.empty(len(g2d), dtype=torch.float64, device=xtd.device)
    ptrs = (ctypes.c_void_p * len(g2d))(*[g.data_ptr() for g in g2d])
    wsb = _lib.query("lddmm_metric_dots_%s_workspace" % sfx, n, d, T, len(g2d))
    ws = workspace.get(wsb)
    _lib.call("lddmm_metric_dots_" + sfx, ptr(xtd), n, d, T, ptr(g1d), ctypes.cast(ptrs, ctypes.c_void_p), len(g2d),
              sigma, order, ptr(out),
              ptr(ws), wsb, stream_handle())
    return out


def covector(xt, at, px1, KparDiff, regweight, with_dat=True, dt=None):
    """Device call: returns (pxt, dat) given the trajectory xt (T+1, N, dim); dt defaults to 1/T."""
    require_cuda()
    xtd, atd, pxd = to_dev(xt), to_dev(at), to_dev(px1)
    T, n, d = atd.shape
    sigma, order, sfx = _kernel_args(KparDiff)
    pxt = torch.empty((T + 1, n, d), dtype=torch.float64, device=xtd.device)
    dat = torch.empty((T, n, d), dtype=torch.float64, device=xtd.device) if with_dat else None
    wsb = _lib.query("lddmm_covector_%s_workspace" % sfx, n, d, T)
    ws = workspace.get(wsb)
    _lib.call("lddmm_covector_" + sfx, ptr(xtd), n, d, ptr(atd), T, float(dt or 0.0), ptr(pxd), sigma, order,
              float(regweight),
              ptr(pxt), ptr(dat) if dat is not None else None, ptr(ws), wsb, stream_handle())
    return pxt, dat


def landmarkDirectEvolutionEuler(x0, at, KparDiff, affine=None, withJacobian=False, withNormals=None,
                                 withPointSet=None):
    """Solves dx/dt = K(x,x) a(t) with x(0) = x0 (pointEvolution.py:662-730)."""
    _check_affine(affine)
    if withNormals is None and withPointSet is None and not withJacobian:
        xt, _ = shoot(x0, at, KparDiff)
        return output_like(x0, xt)
    require_cuda()
    x0d, atd = to_dev(x0), to_dev(at)
    M = atd.shape[0] + 1
    timeStep = 1.0 / (M - 1)
    xt, _ = shoot(x0d, atd, KparDiff)
    out = [xt]
    if withPointSet is not None:
        yt = torch.empty((M,) + tuple(to_dev(withPointSet).shape), dtype=torch.float64, device=x0d.device)
        yt[0] = to_dev(withPointSet)
        if withJacobian:
            Jt = torch.zeros((M, yt.shape[1]), dtype=torch.float64, device=x0d.device)
    elif withJacobian:
        Jt = torch.zeros((M, atd.shape[1]), dtype=torch.float64, device=x0d.device)
    if withNormals is not None:
        nt = torch.empty_like(xt)
        nt[0] = to_dev(withNormals)
    for k in range(M - 1):
        z, a = xt[k], atd[k]
        if withPointSet is not None:
            yt[k + 1] = yt[k] + timeStep * KparDiff.applyK(z, a, firstVar=yt[k])
            if withJacobian:
                Jt[k + 1] = Jt[k] + timeStep * KparDiff.applyDivergence(z, a, firstVar=yt[k])
        elif withJacobian:
            Jt[k + 1] = Jt[k] + timeStep * KparDiff.applyDivergence(z, a)
        if withNormals is not None:
            nt[k + 1] = nt[k] - timeStep * KparDiff.applyDiffKT(z, nt[k][None], a[None])
    if withPointSet is not None:
        out.append(yt)
    if withNormals is not None:
        out.append(nt)
    if withJacobian:
        out.append(Jt)
    return [output_like(x0, t) for t in out]


def landmarkEPDiff(T, x0, a0, KparDiff, affine=None, withJacobian=False, withNormals=None, withPointSet=None):
    """Momentum-carrying (EPDiff) shooting (pointEvolution.py:599-658); returns (xt, at), or
    [xt, at, yt?, nt?, Jt?] with the optional outputs in the reference's order:
      yt[k+1] = yt[k] + dt K(yt[k], x_k) a_k                        (withPointSet)
      nt[k+1] = nt[k] - dt applyDiffKT(x_k, [nt[k]], [a_k])          (withNormals)
      Jt[k+1] = Jt[k] + dt applyDivergence(x_k, a_k)                 (withJacobian; on the
                points x, also with a point set, as in the reference: Jt is (T+1, N))"""
    _check_affine(affine)
    xt, at = _epdiff(T, x0, a0, KparDiff)
    if not withJacobian and withNormals is None and withPointSet is None:
        return output_like(x0, xt), output_like(x0, at)
    timeStep = 1.0 / T
    out = [xt, at]
    if withPointSet is not None:
        y0 = to_dev(withPointSet)
        yt = torch.empty((T + 1,) + tuple(y0.shape), dtype=torch.float64, device=xt.device)
        yt[0] = y0
    if withNormals is not None:
        nt = torch.empty_like(xt)
        nt[0] = to_dev(withNormals)
    if withJacobian:
        Jt = torch.zeros((T + 1, xt.shape[1]), dtype=torch.float64, device=xt.device)
    for k in range(T):
        z, a = xt[k], at[k]
        if withPointSet is not None:
            yt[k + 1] = yt[k] + timeStep * KparDiff.applyK(z, a, firstVar=yt[k])
        if withNormals is not None:
            nt[k + 1] = nt[k] - timeStep * KparDiff.applyDiffKT(z, nt[k][None], a[None])
        if withJacobian:
            Jt[k + 1] = Jt[k] + timeStep * KparDiff.applyDivergence(z, a)
    if withPointSet is not None:
        out.append(yt)
    if withNormals is not None:
        out.append(nt)
    if withJacobian:
        out.append(Jt)
    return [output_like(x0, t) for t in out]


def _epdiff(T, x0, a0, KparDiff):
    """The fused EPDiff operator (lddmm_epdiff_*): device (xt, at)."""
    require_cuda()
    x0d, a0d = to_dev(x0), to_dev(a0)
    n, d = x0d.shape
    sigma, order, sfx = _kernel_args(KparDiff)
    xt = torch.empty((T + 1, n, d), dtype=torch.float64, device=x0d.device)
    at = torch.zeros((T, n, d), dtype=torch.float64, device=x0d.device)
    wsb = _lib.query("lddmm_epdiff_%s_workspace" % sfx, n, d, T)
    ws = workspace.get(wsb)
    _lib.call("lddmm_epdiff_" + sfx, ptr(x0d), n, d, ptr(a0d), int(T), sigma, order, ptr(xt), ptr(at), ptr(ws), wsb,
              stream_handle())
    return xt, at


def landmarkHamiltonianCovector(x0, at, px1, KparDiff, regweight, affine=None):
    """Re-shoots, then integrates the covector backwards (pointEvolution.py:735-765); returns (pxt, xt)."""
    _check_affine(affine)
    xt, _ = shoot(x0, at, KparDiff)
    pxt, _ = covector(xt, at, px1, KparDiff, regweight, with_dat=False)
    return output_like(x0, pxt), output_like(x0, xt)


def landmarkHamiltonianGradient(x0, at, px1, KparDiff, regweight, getCovector=False, affine=None):
    """dat_k = 2 rw a_k - p_{k+1} (pointEvolution.py:793-817).  Returns (dat, xt[, pxt]);
    with a (zero) affine argument the reference also returns zero dA, db."""
    _check_affine(affine)
    xt, _ = shoot(x0, at, KparDiff)
    pxt, dat = covector(xt, at, px1, KparDiff, regweight, with_dat=True)
    dat_o, xt_o, pxt_o = output_like(x0, dat), output_like(x0, xt), output_like(x0, pxt)
    if affine is None:
        return (dat_o, xt_o, pxt_o) if getCovector else (dat_o, xt_o)
    dA = np.zeros(np.shape(affine[0])) if not is_device(x0) else torch.zeros_like(to_dev(affine[0]))
    db = np.zeros(np.shape(affine[1])) if not is_device(x0) else torch.zeros_like(to_dev(affine[1]))
    return (dat_o, dA, db, xt_o, pxt_o) if getCovector else (dat_o, dA, db, xt_o)


def secondOrderEvolution(x0, a0, rhot, KparDiff, withJacobian=False, withPointSet=None, affine=None):
    """x_{k+1} = x_k + dt K(x_k) a_k,  a_{k+1} = a_k + dt (-applyDiffKT(x_k, [a_k], [a_k]) + rho_k)
    (pointEvolution.py:882-951); returns (xt, at), or [xt, at, zt(, Jt)] with a point set.
    The reference's withJacobian without a point set reads undefined names; it is rejected."""
    _check_affine(affine)
    if withJacobian and withPointSet is None:
        raise NotImplementedError("withJacobian needs withPointSet (the reference's other branch is undefined)")
    require_cuda()
    x0d, a0d, rho = to_dev(x0), to_dev(a0), to_dev(rhot)
    T = rho.shape[0]
    dt = 1.0 / T
    xt = torch.empty((T + 1,) + tuple(x0d.shape), dtype=torch.float64, device=x0d.device)
    at = torch.empty_like(xt)
    xt[0], at[0] = x0d, a0d
    if withPointSet is not None:
        z0 = to_dev(withPointSet)
        zt = torch.empty((T + 1,) + tuple(z0.shape), dtype=torch.float64, device=x0d.device)
        zt[0] = z0
        if withJacobian:
            Jt = torch.zeros((T + 1, z0.shape[0]), dtype=torch.float64, device=x0d.device)
    for k in range(T):
        x, a = xt[k], at[k]
        zx = KparDiff.applyK(x, a)
        za = -KparDiff.applyDiffKT(x, a[None], a[None]) + rho[k]
        xt[k + 1] = x + dt * zx
        at[k + 1] = a + dt * za
        if withPointSet is not None:
            zt[k + 1] = zt[k] + dt * KparDiff.applyK(x, a, firstVar=zt[k])
            if withJacobian:
                Jt[k + 1] = Jt[k] + dt * KparDiff.applyDivergence(x, a, firstVar=zt[k])
    if withPointSet is None:
        return output_like(x0, xt), output_like(x0, at)
    out = [xt, at, zt] + ([Jt] if withJacobian else [])
    return [output_like(x0, t) for t in out]


def secondOrderHamiltonian(x, a, rho, px, pa, KparDiff, affine=None):
    """<px, K a> + <pa, -applyDiffKT(x, [a], [a]) + rho> - |rho|^2 / 2 (pointEvolution.py:954-964)."""
    _check_affine(affine)
    xd, ad, rd, pxd, pad = (to_dev(v) for v in (x, a, rho, px, pa))
    Ht = (pxd * KparDiff.applyK(xd, ad)).sum()
    Ht = Ht + (pad * (-KparDiff.applyDiffKT(xd, ad[None], ad[None]) + rd)).sum()
    Ht = Ht - (rd ** 2).sum() / 2
    return float(Ht)


def secondOrderCovector(x0, a0, rhot, px1, pa1, KparDiff, affine=None, times=None):
    """Backward adjoint of the second-order evolution (pointEvolution.py:967-1043):
      px_t = px_{t+1} + dt (applyDiffKT(x, [px, a], [a, px]) - applyDDiffK11and12(x, a, a, pa)),
      pa_t = pa_{t+1} + dt (applyK(x, px) - applyDiffK1and2(x, pa, a)),
    with the target terms px1[j], pa1[j] added at the intermediate times.  Returns
    (pxt, pat, xt, at).  (The reference's `times=None` branch builds an unused
    array from `range(nTarg) + 1`, which raises; it is skipped.)"""
    _check_affine(affine)
    require_cuda()
    rho = to_dev(rhot)
    T = rho.shape[0]
    P1 = [to_dev(v) for v in px1]
    A1 = [to_dev(v) for v in pa1]
    nTarg = len(P1)
    Tsize1 = T // nTarg
    dt = 1.0 / T
    xt, at = secondOrderEvolution(to_dev(x0), to_dev(a0), rho, KparDiff)
    pxt = torch.zeros_like(xt)
    pat = torch.zeros_like(xt)
    pxt[T], pat[T] = P1[nTarg - 1], A1[nTarg - 1]
    for t in range(T):
        px, pa = pxt[T - t], pat[T - t]
        x, a = xt[T - t - 1], at[T - t - 1]
        zpx = KparDiff.applyDiffKT(x, torch.stack([px, a]), torch.stack([a, px])) \
            - KparDiff.applyDDiffK11and12(x, a, a, pa)
        zpa = KparDiff.applyK(x, px) - KparDiff.applyDiffK1and2(x, pa, a)
        pxt[T - t - 1] = px + dt * zpx
        pat[T - t - 1] = pa + dt * zpa
        if t < T - 1 and (T - 1 - t) % Tsize1 == 0:
            pxt[T - t - 1] += P1[(T - t - 1) // Tsize1 - 1]
            pat[T - t - 1] += A1[(T - t - 1) // Tsize1 - 1]
    return tuple(output_like(x0, v) for v in (pxt, pat, xt, at))


def secondOrderGradient(x0, a0, rhot, px1, pa1, KparDiff, times=None, getCovector=False, affine=None,
                        controlWeight=1.0):
    """da0 = K(x0) a0 - pa_0 (pointEvolution.py:1046-1091).  Without affine the
    reference returns drhot = 0 (its rho - pa line is commented out); kept.
    Returns (da0, drhot, xt, at[, pxt, pat]); affine=None only."""
    if affine is not None:
        raise NotImplementedError("affine second-order gradients are not provided (affine=None only)")
    pxt, pat, xt, at = secondOrderCovector(to_dev(x0), to_dev(a0), to_dev(rhot), px1, pa1, KparDiff, times=times)
    drhot = torch.zeros_like(to_dev(rhot))
    da0 = KparDiff.applyK(to_dev(x0), to_dev(a0)) - pat[0]
    out = (da0, drhot, xt, at) + ((pxt, pat) if getCovector else ())
    return tuple(output_like(x0, to_dev(v)) for v in out)

