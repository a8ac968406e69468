"""Drop-in for the f2py module ``kernelFunctions_fort`` of py-lddmm, on the GPU.

py-lddmm's kernelFunctions.py binds its native loops with
``import kernelFunctions_fort as kff`` (kernelFunctions.py:2) and calls them
with f2py's positional argument lists (kernelFunctions.py:318-327, 391-455).
This module has the same names and argument lists, numpy in and numpy out,
and computes on the GPU through liblddmm_b200.so.  Making the reference run
on it takes one line before its modules are imported::

    import sys
    from registration_b200 import kernelFunctions_fort
    sys.modules["kernelFunctions_fort"] = kernelFunctions_fort

f2py conventions kept (the wrappers that f2py generates from
kernelFunctions.f90):

* array arguments are converted to FP64 (any array-like, lists included);
* the trailing size arguments (num_nodes, num_nodes_y, dim, dimb, na) may be
  given or left out; given, they must agree with the arrays' shapes, and a
  disagreement raises ValueError before any GPU work;
* ``ord > 4`` selects the Gaussian kernel, 0..4 the Laplacian (Matern) order;
* the result is a fresh Fortran-ordered float64 array; calls are synchronous.

Precision: kernel sums in FP32 with compensated (TwoSum) accumulation and FP64
results by default ('fp32c'); ``set_precision('fp64')`` selects plain FP64 on
the GPU (what the Fortran computes).  The environment variable
LDDMM_KFF_PRECISION sets the initial value.  There is no CPU fallback: without
a CUDA device or the library every call raises.
"""
import os

import numpy as np

from . import kernelFunctions as _kf

__all__ = ["applyk", "applykdifft", "applykmat", "applykdiffmat", "applykdiff1", "applykdiff2", "applykdiff1and2",
           "applykdiff11", "applykdiff12", "applykdiff11and12", "set_precision", "get_precision"]

_precision = os.environ.get("LDDMM_KFF_PRECISION", "fp32c")
if _precision not in _kf.PRECISIONS:
    raise ValueError("LDDMM_KFF_PRECISION must be one of %s" % (_kf.PRECISIONS,))
_kernels = {}


def set_precision(precision):
    """'fp32c' (default) or 'fp64' for every following call."""
    global _precision
    if precision not in _kf.PRECISIONS:
        raise ValueError("precision must be one of %s" % (_kf.PRECISIONS,))
    _precision = precision


def get_precision():
    return _precision


def _kernel(sig, ord_):
    """The kernel of the Fortran (sig, ord) pair: ord > 4 is the Gaussian."""
    ord_ = int(ord_)
    if ord_ < 0:
        raise ValueError("ord must be >= 0")
    key = (float(sig), ord_ if ord_ <= 4 else 10, _precision)
    K = _kernels.get(key)
    if K is None:
        K = _kf.Kernel(name="gauss" if ord_ > 4 else "laplacian", sigma=float(sig), order=key[1],
                       precision=_precision)
        _kernels[key] = K
    return K


def _arr(a, name, ndim):
    t = np.asarray(a, dtype=np.float64)
    if t.ndim != ndim:
        raise ValueError("%s: expected a rank-%d array, got shape %s" % (name, ndim, t.shape))
    return np.ascontiguousarray(t)


def _agree(name, given, actual):
    if given is not None and int(given) != int(actual):
        raise ValueError("%s = %d does not match the array extent %d" % (name, int(given), int(actual)))


def _out(f):
    return np.asfortranarray(f)


def applyk(x, y, beta, sig, ord, num_nodes=None, num_nodes_y=None, dim=None, dimb=None):
    """f[k] = sum_l K(x_k, y_l) beta_l (kernelFunctions.f90:1-54)."""
    x, y, beta = _arr(x, "x", 2), _arr(y, "y", 2), _arr(beta, "beta", 2)
    _agree("num_nodes", num_nodes, x.shape[0])
    _agree("num_nodes_y", num_nodes_y, y.shape[0])
    _agree("dim", dim, x.shape[1])
    _agree("dimb", dimb, beta.shape[1])
    if y.shape[1] != x.shape[1] or beta.shape[0] != y.shape[0]:
        raise ValueError("applyk: x (%s), y (%s) and beta (%s) do not agree" % (x.shape, y.shape, beta.shape))
    return _out(_kernel(sig, ord).applyK(y, beta, firstVar=x))


def applykdifft(x, y, a1, a2, sig, ord, num_nodes=None, num_nodes_y=None, dim=None, dimb=None, na=None):
    """f[k] = sum_l K'(x_k, y_l) 2 (x_k - y_l) sum_{i,c} a1[i,k,c] a2[i,l,c]
    (kernelFunctions.f90:56-114)."""
    x, y, a1, a2 = _arr(x, "x", 2), _arr(y, "y", 2), _arr(a1, "a1", 3), _arr(a2, "a2", 3)
    _agree("num_nodes", num_nodes, x.shape[0])
    _agree("num_nodes_y", num_nodes_y, y.shape[0])
    _agree("dim", dim, x.shape[1])
    _agree("dimb", dimb, a1.shape[2])
    _agree("na", na, a1.shape[0])
    if (y.shape[1] != x.shape[1] or a1.shape[1] != x.shape[0] or a2.shape[1] != y.shape[0]
            or a1.shape[0] != a2.shape[0] or a1.shape[2] != a2.shape[2]):
        raise ValueError("applykdifft: x (%s), y (%s), a1 (%s) and a2 (%s) do not agree"
                         % (x.shape, y.shape, a1.shape, a2.shape))
    return _out(_kernel(sig, ord).applyDiffKT(y, a1, a2, firstVar=x))


def applykmat(x, y, beta, sig, ord, num_nodes=None, num_nodes_y=None, dim=None, dimb=None):
    """f[k] = sum_l K(x_k, y_l) beta[k, l, :] (kernelFunctions.f90:499-552)."""
    x, y, beta = _arr(x, "x", 2), _arr(y, "y", 2), _arr(beta, "beta", 3)
    _agree("num_nodes", num_nodes, x.shape[0])
    _agree("num_nodes_y", num_nodes_y, y.shape[0])
    _agree("dim", dim, x.shape[1])
    _agree("dimb", dimb, beta.shape[2])
    if y.shape[1] != x.shape[1] or beta.shape[:2] != (x.shape[0], y.shape[0]):
        raise ValueError("applykmat: x (%s), y (%s) and beta (%s) do not agree" % (x.shape, y.shape, beta.shape))
    return _out(_kernel(sig, ord).applyK(y, beta, firstVar=x, matrixWeights=True))


def applykdiffmat(x, y, beta, sig, ord, num_nodes=None, num_nodes_y=None, dim=None):
    """f[k] = sum_l K'(x_k, y_l) 2 (x_k - y_l) beta[k, l] (kernelFunctions.f90:554-610)."""
    x, y, beta = _arr(x, "x", 2), _arr(y, "y", 2), _arr(beta, "beta", 2)
    _agree("num_nodes", num_nodes, x.shape[0])
    _agree("num_nodes_y", num_nodes_y, y.shape[0])
    _agree("dim", dim, x.shape[1])
    if y.shape[1] != x.shape[1] or beta.shape != (x.shape[0], y.shape[0]):
        raise ValueError("applykdiffmat: x (%s), y (%s) and beta (%s) do not agree" % (x.shape, y.shape, beta.shape))
    return _out(_kernel(sig, ord).applyDiffKmat(y, beta, firstVar=x))


def _self_pair(routine, x, arrays, sig, ord, num_nodes, dim):
    x = _arr(x, "x", 2)
    arrs = [_arr(a, nm, 2) for nm, a in arrays]
    _agree("num_nodes", num_nodes, x.shape[0])
    _agree("dim", dim, x.shape[1])
    for (nm, _), a in zip(arrays, arrs):
        if a.shape != x.shape:
            raise ValueError("%s: %s (%s) must have the shape of x (%s)" % (routine, nm, a.shape, x.shape))
    return _out(_kernel(sig, ord)._kdiffx(routine, x, *arrs))


def applykdiff1(x, a1, a2, sig, ord, num_nodes=None, dim=None):
    """f_k = sum_l K' 2 <x_k - x_l, a1_k> a2_l (kernelFunctions.f90:116-172)."""
    return _self_pair("applykdiff1", x, [("a1", a1), ("a2", a2)], sig, ord, num_nodes, dim)


def applykdiff2(x, a1, a2, sig, ord, num_nodes=None, dim=None):
    """f_k = -sum_l K' 2 <x_k - x_l, a1_l> a2_l (kernelFunctions.f90:174-230)."""
    return _self_pair("applykdiff2", x, [("a1", a1), ("a2", a2)], sig, ord, num_nodes, dim)


def applykdiff1and2(x, a1, a2, sig, ord, num_nodes=None, dim=None):
    """applykdiff1 + applykdiff2 in one sweep (kernelFunctions.f90:233-290)."""
    return _self_pair("applykdiff1and2", x, [("a1", a1), ("a2", a2)], sig, ord, num_nodes, dim)


def applykdiff11(x, a1, a2, p, sig, ord, num_nodes=None, dim=None):
    """sum_l <a1_k, a2_l> (K'' 4 <dx, p_k> dx + K' 2 p_k) (kernelFunctions.f90:293-359),
    over the intended y = x (the Fortran loops over an undeclared num_nodes_y)."""
    return _self_pair("applykdiff11", x, [("a1", a1), ("a2", a2), ("p", p)], sig, ord, num_nodes, dim)


def applykdiff12(x, a1, a2, p, sig, ord, num_nodes=None, dim=None):
    """-sum_l <a1_k, a2_l> (K'' 4 <dx, p_l> dx + K' 2 p_l) (kernelFunctions.f90:361-428), y = x."""
    return _self_pair("applykdiff12", x, [("a1", a1), ("a2", a2), ("p", p)], sig, ord, num_nodes, dim)


def applykdiff11and12(x, a1, a2, p, sig, ord, num_nodes=None, dim=None):
    """sum_l <a1_k, a2_l> (K'' 4 <dx, p_k - p_l> dx + K' 2 (p_k - p_l)) (kernelFunctions.f90:430-496)."""
    return _self_pair("applykdiff11and12", x, [("a1", a1), ("a2", a2), ("p", p)], sig, ord, num_nodes, dim)
