"""Kernel API with the signatures of py-lddmm/kernelFunctions.py (KernelSpec,
Kernel.applyK / applyDiffKT / applyDiffKmat ...), computed by the CUDA library.

Drop-in rules kept from the reference:
  * ``KernelSpec(name, affine, sigma, order, w1, w2, dim, center, weight)``:
    'gauss' forces order 10, 'laplacian' orders above 4 become 3, any other
    name means "no kernel" (kernelFunctions.py:238-268);
  * ``applyK(x, a, firstVar=None)``: x are the sources, firstVar the targets
    (x itself when None) (kernelFunctions.py:310-330);
  * ``weight`` only scales ``precompute`` (dense matrices), never applyK
    (kernelFunctions.py:285-298);
  * outputs are fresh float64 arrays: numpy in -> numpy out; CUDA tensors in ->
    CUDA tensors out (stays on the device).
Affine kernel parts (``affine='affine'`` or ``'euclidean'``, kernelFunctions.py:
334-367 and 431-448) are added on the device after the kernel sums, from the
FP64 moments of the sources (lddmm_moments_f64, lddmm_rows_affine_f64).

Extra keyword: ``precision`` = 'fp32c' (default: FP32 pair arithmetic with
compensated accumulation, FP64 results) or 'fp64' (plain FP64 on the GPU).
"""
import numpy as np
import torch

from . import _lib
from .device import output_like, ptr, require_cuda, stream_handle, to_dev, workspace

PRECISIONS = ("fp32c", "fp64")


def _suffix(precision):
    if precision not in PRECISIONS:
        raise ValueError("precision must be one of %s" % (PRECISIONS,))
    return "f32c" if precision == "fp32c" else "f64"


class KernelSpec:
    """Kernel parameters (kernelFunctions.py:238-280)."""

    def __init__(self, name='gauss', affine='none', sigma=6.5, order=10, w1=1.0, w2=1.0, dim=3, center=(0, 0, 0),
                 weight=1.0, precision='fp32c'):
        self.name = name
        self.sigma = sigma
        self.order = order
        self.weight = weight
        self.w1 = w1
        self.w2 = w2
        self.constant_plane = False
        self.center = np.array(center)
        self.affine_basis = []
        self.dim = dim
        self.precomp = []
        self._hold = False
        self._state = False
        self.affine = affine
        self.precision = precision
        _suffix(precision)
        if name == 'laplacian':
            if self.order > 4:
                self.order = 3
            self.par = [sigma, self.order]
        elif name == 'gauss':
            self.order = 10
            self.par = [sigma]
        else:
            self.name = 'none'
            self.par = []
        if affine is None:
            self.affine = 'none'
        elif affine not in ('none', 'affine', 'euclidean'):
            raise ValueError("affine must be 'none', 'affine' or 'euclidean'")
        if self.affine == 'euclidean':
            # the skew-symmetric basis of the reference (kernelFunctions.py:268-278)
            s2 = np.sqrt(2.0)
            if dim == 3:
                self.affine_basis = [np.array([[0, 1, 0], [-1, 0, 0], [0, 0, 0]]) / s2,
                                     np.array([[0, 0, 1], [0, 0, 0], [-1, 0, 0]]) / s2,
                                     np.array([[0, 0, 0], [0, 0, 1], [0, -1, 0]]) / s2]
            elif dim == 2:
                self.affine_basis = [np.array([[0, 1], [-1, 0]]) / s2]
            else:
                raise ValueError("euclidean kernels are available in dimension 2 or 3 only")


class Kernel(KernelSpec):
    """Kernel with the apply* methods of kernelFunctions.py:284-530."""

    # hold/release/reset keep the reference's state machine (kernelFunctions.py:300-307);
    # no dense matrix is cached, so they have no numerical effect.
    def hold(self):
        self._state = self._hold
        self._hold = True

    def release(self):
        self._state = False
        self._hold = False

    def reset(self):
        self._hold = self._state

    # ---- kernel sums -----------------------------------------------------
    def applyK(self, x, a, firstVar=None, grid=None, matrixWeights=False):
        """K(x, x) a, or K(firstVar, x) a (kernelFunctions.py:310-369)."""
        if matrixWeights:
            return self._applykmat(x, a, firstVar)
        require_cuda()
        src = to_dev(x)
        w = to_dev(a)
        tgt = src if firstVar is None else to_dev(firstVar)
        if w.dim() != 2 or w.shape[0] != src.shape[0]:
            raise ValueError("applyK: a must be (N, dimb) with N = x.shape[0]")
        n, m, d, dimb = tgt.shape[0], src.shape[0], src.shape[1], w.shape[1]
        if tgt.shape[1] != d:
            raise ValueError("applyK: firstVar and x have different dimensions")
        if self.name == 'none':
            f = torch.zeros((n, dimb), dtype=torch.float64, device=src.device)
        else:
            f = torch.empty((n, dimb), dtype=torch.float64, device=src.device)
            sfx = _suffix(self.precision)
            wsb = _lib.query("lddmm_applyk_%s_workspace" % sfx, n, m, d, dimb)
            ws = workspace.get(wsb)
            _lib.call("lddmm_applyk_" + sfx, ptr(tgt), n, ptr(src), m, ptr(w), d, dimb, float(self.sigma),
                      int(self.order), ptr(f), ptr(ws), wsb, stream_handle())
        if self.affine != 'none':
            self._affine_applyk(src, w, tgt, f)
        return output_like(x, f)

    # ---- affine parts (kernelFunctions.py:334-367, 431-448) -------------------
    def _center_dev(self, d, device):
        c = np.zeros(d)
        cc = np.asarray(self.center, dtype=np.float64).reshape(-1)
        c[:min(d, cc.size)] = cc[:d]
        return torch.from_numpy(c).to(device)

    def _moments(self, src, w, c):
        """(M, s) on the host: M = sum_l (x_l - c) w_l^T (d x dimb), s = sum_l w_l (FP64 on the device)."""
        m, d = src.shape
        dimb = w.shape[1]
        out = torch.empty(d * dimb + dimb, dtype=torch.float64, device=src.device)
        wsb = _lib.query("lddmm_moments_f64_workspace", m, d, dimb)
        ws = workspace.get(wsb)
        _lib.call("lddmm_moments_f64", ptr(src), m, d, ptr(w.contiguous()), dimb, ptr(c), ptr(out), ptr(ws), wsb,
                  stream_handle())
        h = out.cpu().numpy()
        return h[:d * dimb].reshape(d, dimb), h[d * dimb:]

    def _rows(self, u, c, W, b, f):
        """f += (u - c) W + b on the device (lddmm_rows_affine_f64)."""
        n, Q = u.shape
        J = f.shape[1]
        Wd = torch.from_numpy(np.ascontiguousarray(W, dtype=np.float64)).to(f.device)
        bd = None if b is None else torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).to(f.device)
        _lib.call("lddmm_rows_affine_f64", ptr(u.contiguous()), n, Q, ptr(c) if c is not None else None, ptr(Wd),
                  ptr(bd) if bd is not None else None, J, ptr(f), stream_handle())

    def _affine_applyk(self, src, w, tgt, f):
        d = src.shape[1]
        if w.shape[1] > 4:
            raise ValueError("affine kernel parts need at most 4 weight columns")
        c = self._center_dev(d, src.device)
        M, sums = self._moments(src, w, c)
        if self.affine == 'affine':
            # z += w1 (y - c) ((x - c)^T a) + w2 sum_l a_l
            W = self.w1 * M
        else:
            if w.shape[1] != d:
                raise ValueError("euclidean kernel parts need weights of the points' dimension")
            # z += w2 sum_l a_l + w1 sum_E <(x - c) E^T, a> (y - c) E^T
            W = np.zeros((d, d))
            for E in self.affine_basis:
                W += self.w1 * float((E * M.T).sum()) * E.T
        self._rows(tgt, c, W, self.w2 * sums, f)

    def _affine_difft(self, src, A1, A2, tgt, f):
        if self.affine == 'affine':
            # the reference's branch reads an undefined variable (kernelFunctions.py:437)
            raise NotImplementedError("applyDiffKT of an 'affine' kernel fails in the reference "
                                      "(kernelFunctions.py:437 uses an undefined `a`)")
        na, _, d = A1.shape
        c = self._center_dev(d, src.device)
        # zpx += w1 sum_E sum_k <(x - c) E^T, a2[k]> a1[k] E
        Bs = []
        for k in range(na):
            Mk, _ = self._moments(src, A2[k], c)
            B = np.zeros((d, d))
            for E in self.affine_basis:
                B += float((E * Mk.T).sum()) * E
            Bs.append(self.w1 * B)
        step = max(1, 16 // d)
        for k0 in range(0, na, step):
            ks = list(range(k0, min(na, k0 + step)))
            u = torch.cat([A1[k] for k in ks], dim=1)
            self._rows(u, None, np.concatenate([Bs[k] for k in ks], axis=0), None, f)

    def applyDiffKT(self, x, a1, a2, firstVar=None):
        """sum_l grad_1 [a1_k . K(y_k, x_l) a2_l] (kernelFunctions.py:412-449)."""
        require_cuda()
        src = to_dev(x)
        tgt = src if firstVar is None else to_dev(firstVar)
        A1 = _stack(a1)
        A2 = _stack(a2)
        if A1.dim() != 3 or A2.dim() != 3 or A1.shape[0] != A2.shape[0] or A1.shape[2] != A2.shape[2]:
            raise ValueError("applyDiffKT: a1, a2 must be (na, N, dimb) with matching na and dimb")
        na, dimb = A1.shape[0], A1.shape[2]
        n, m, d = tgt.shape[0], src.shape[0], src.shape[1]
        if A1.shape[1] != n or A2.shape[1] != m:
            raise ValueError("applyDiffKT: a1 must cover the targets and a2 the sources")
        if self.affine != 'none':
            if self.affine == 'euclidean' and dimb != d:
                raise ValueError("euclidean kernel parts need momenta of the points' dimension")
            plain = self._plain()
            f = to_dev(plain.applyDiffKT(src, A1, A2, firstVar=None if firstVar is None else tgt))
            f = f.clone()
            self._affine_difft(src, A1, A2, tgt, f)
            return output_like(x, f)
        if self.name == 'none':
            return output_like(x, torch.zeros((n, d), dtype=torch.float64, device=src.device))
        f = torch.empty((n, d), dtype=torch.float64, device=src.device)
        sfx = _suffix(self.precision)
        if na * dimb > 12:
            # linear in the (i, c) terms: accumulate groups of whole momenta
            step = max(1, 12 // dimb)
            acc = None
            for i0 in range(0, na, step):
                part = self.applyDiffKT(src, A1[i0:i0 + step], A2[i0:i0 + step],
                                        firstVar=None if firstVar is None else tgt)
                acc = part if acc is None else acc + part
            return output_like(x, acc)
        wsb = _lib.query("lddmm_applykdifft_%s_workspace" % sfx, n, m, na, d, dimb)
        ws = workspace.get(wsb)
        _lib.call("lddmm_applykdifft_" + sfx, ptr(tgt), n, ptr(src), m, ptr(A1), ptr(A2), na, d, dimb,
                  float(self.sigma), int(self.order), ptr(f), ptr(ws), wsb, stream_handle())
        return output_like(x, f)

    def _plain(self):
        """The same kernel without its affine part."""
        K = Kernel(name=self.name, sigma=self.sigma, order=self.order, weight=self.weight, precision=self.precision)
        K.name = self.name
        return K

    def applyDivergence(self, x, a, firstVar=None):
        """sum_l div_1 K(y_k, x_l) a_l, times KernelSpec.weight as the dense
        precompute path of the reference (kernelFunctions.py:509-530)."""
        require_cuda()
        src = to_dev(x)
        w = to_dev(a)
        tgt = src if firstVar is None else to_dev(firstVar)
        n, m, d = tgt.shape[0], src.shape[0], src.shape[1]
        if self.name == 'none':
            return output_like(x, torch.zeros(n, dtype=torch.float64, device=src.device))
        f = torch.empty(n, dtype=torch.float64, device=src.device)
        sfx = _suffix(self.precision)
        wsb = _lib.query("lddmm_applydiv_%s_workspace" % sfx, n, m, d)
        ws = workspace.get(wsb)
        _lib.call("lddmm_applydiv_" + sfx, ptr(tgt), n, ptr(src), m, ptr(w), d, float(self.sigma), int(self.order),
                  ptr(f), ptr(ws), wsb, stream_handle())
        if self.weight != 1.0:
            f = f * self.weight
        return output_like(x, f)

    # ---- first / second derivative loops (kernelFunctions.f90:116-496) -----------
    _KDIFF_ROUTINES = {"applykdiff1": 1, "applykdiff2": 2, "applykdiff1and2": 3, "applykdiff11": 11,
                       "applykdiff12": 12, "applykdiff11and12": 13}

    def _kdiffx(self, routine, x, a1, a2, p=None):
        require_cuda()
        xd, A1, A2 = to_dev(x), to_dev(a1), to_dev(a2)
        n, d = xd.shape
        for t in (A1, A2) + ((to_dev(p),) if p is not None else ()):
            if tuple(t.shape) != (n, d):
                raise ValueError("%s: a1, a2 (and p) must be (N, dim) like x" % routine)
        if self.name == 'none':
            return output_like(x, torch.zeros((n, d), dtype=torch.float64, device=xd.device))
        f = torch.empty((n, d), dtype=torch.float64, device=xd.device)
        sfx = _suffix(self.precision)
        wsb = _lib.query("lddmm_applykdiffx_%s_workspace" % sfx, self._KDIFF_ROUTINES[routine], n, d, int(self.order))
        ws = workspace.get(wsb)
        args = [ptr(xd), n, d, ptr(A1.contiguous()), ptr(A2.contiguous())]
        if p is not None:
            args.append(ptr(to_dev(p).contiguous()))
        _lib.call("lddmm_%s_%s" % (routine, sfx), *args, float(self.sigma), int(self.order), ptr(f), ptr(ws), wsb,
                  stream_handle())
        return output_like(x, f)

    def applyDiffK(self, x, a1, a2):
        """A_k = sum_l K'(x_k, x_l) 2 <x_k - x_l, a1_k> a2_l (kernelFunctions.py:391-393 -> kff.applykdiff1)."""
        return self._kdiffx("applykdiff1", x, a1, a2)

    def applyDiffK2(self, x, a1, a2):
        """A_k = -sum_l K' 2 <x_k - x_l, a1_l> a2_l (kernelFunctions.py:396-398 -> kff.applykdiff2)."""
        return self._kdiffx("applykdiff2", x, a1, a2)

    def applyDiffK1and2(self, x, a1, a2):
        """applyDiffK + applyDiffK2 in one sweep (kernelFunctions.py:400-402 -> kff.applykdiff1and2)."""
        return self._kdiffx("applykdiff1and2", x, a1, a2)

    def applyDDiffK11and12(self, x, n, a, p):
        """sum_l D_11 + D_12 of n_k^T K(x_k, x_l) a_l applied to p (kernelFunctions.py:452-455 ->
        kff.applykdiff11and12)."""
        return self._kdiffx("applykdiff11and12", x, n, a, p)

    def applyDDiffK11(self, x, n, a, p):
        """sum_l D_11[n_k^T K(x_k, x_l) a_l] p_k (kernelFunctions.py:459-478, a dense precompute in the
        reference, hence scaled by KernelSpec.weight; here the applykdiff11 loop)."""
        f = self._kdiffx("applykdiff11", x, n, a, p)
        return f * self.weight if self.weight != 1.0 else f

    def applyDDiffK12(self, x, n, a, p):
        """sum_l D_12[n_k^T K(x_k, x_l) a_l] p_l (kernelFunctions.py:481-507, dense precompute in the
        reference, scaled by KernelSpec.weight; affine='none')."""
        f = self._kdiffx("applykdiff12", x, n, a, p)
        return f * self.weight if self.weight != 1.0 else f

    def _applykmat(self, x, a, firstVar):
        """f_k = sum_l K(y_k, x_l) a[k, l, :] with dense weights a (N_targets, N, dimb)
        (kernelFunctions.py:310-329 -> kff.applykmat, kernelFunctions.f90:499-552)."""
        require_cuda()
        src = to_dev(x)
        tgt = src if firstVar is None else to_dev(firstVar)
        w = to_dev(a)
        n, m, d = tgt.shape[0], src.shape[0], src.shape[1]
        if w.dim() != 3 or w.shape[0] != n or w.shape[1] != m:
            raise ValueError("applyK(matrixWeights=True): a must be (N_targets, N_sources, dimb)")
        dimb = w.shape[2]
        if self.name == 'none':
            return output_like(x, torch.zeros((n, dimb), dtype=torch.float64, device=src.device))
        f = torch.empty((n, dimb), dtype=torch.float64, device=src.device)
        _lib.call("lddmm_applykmat_" + _suffix(self.precision), ptr(tgt), n, ptr(src), m, ptr(w.contiguous()), d,
                  dimb, float(self.sigma), int(self.order), ptr(f), stream_handle())
        return output_like(x, f)

    def applyDiffKmat(self, x, beta, firstVar=None):
        """f_k = sum_l K'(y_k, x_l) 2 (y_k - x_l) beta[k, l] with dense beta (N_targets, N)
        (kernelFunctions.py:405-410 -> kff.applykdiffmat, kernelFunctions.f90:554-610)."""
        require_cuda()
        src = to_dev(x)
        tgt = src if firstVar is None else to_dev(firstVar)
        b = to_dev(beta)
        n, m, d = tgt.shape[0], src.shape[0], src.shape[1]
        if b.dim() != 2 or b.shape[0] != n or b.shape[1] != m:
            raise ValueError("applyDiffKmat: beta must be (N_targets, N_sources)")
        if self.name == 'none':
            return output_like(x, torch.zeros((n, d), dtype=torch.float64, device=src.device))
        f = torch.empty((n, d), dtype=torch.float64, device=src.device)
        _lib.call("lddmm_applykdiffmat_" + _suffix(self.precision), ptr(tgt), n, ptr(src), m, ptr(b.contiguous()),
                  d, float(self.sigma), int(self.order), ptr(f), stream_handle())
        return output_like(x, f)


def _stack(a):
    if isinstance(a, (list, tuple)):
        return torch.stack([to_dev(t) for t in a]).contiguous()
    t = to_dev(a)
    return t
