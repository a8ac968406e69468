"""Oracle -- TEST INFRASTRUCTURE ONLY.

FP64 CPU restatement of the py-lddmm point-LDDMM hot path, used as the checker
by the parity tests, by ``__graft_entry__.smoke()`` and by the CPU baseline /
reference arm of ``bench.py``.  The product package (``registration_b200``)
never imports anything from here.

* ``oracle/kernel_loops.c`` (built into ``liblddmm_oracle.so`` by
  ``oracle/Makefile``) restates the f2py Fortran loops of
  py-lddmm/kernelFunctions.f90 in C/OpenMP.
* ``oracle.lddmm_ref`` is a Python-3 numpy transliteration of the layers above
  (py-lddmm/kernelFunctions.py Kernel, pointEvolution.py landmark*,
  surfaces.py / curves.py norms, surfaceMatching.py, curveMatching.py,
  conjugateGradient.py, gradientDescent.py) calling those loops.

Parity pinning: the reference cannot be built here (no Fortran compiler, no
Python 2), so ``tests/golden/make_golden.py`` runs the reference's own Python
modules (mechanically made Python-3 parseable) on top of this oracle's loops,
and checks the loops themselves against the reference's dense numpy kernel
matrices (kernelMatrixGauss / kernelMatrixLaplacian); the fixtures it writes
pin this oracle.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblddmm_oracle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.c_int64
_int = ctypes.c_int
_dbl = ctypes.c_double


def build(force=False):
    """Compile liblddmm_oracle.so with oracle/Makefile (gcc, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "kernel_loops.c"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "all"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.lddmm_oracle_applyk.argtypes = [_D, _D, _D, _dbl, _int, _i64, _i64, _int, _int, _D]
        L.lddmm_oracle_applykdifft.argtypes = [_D, _D, _D, _D, _dbl, _int, _i64, _i64, _int, _int, _int, _D]
        for nm in ("applykdiff1", "applykdiff2", "applykdiff1and2"):
            getattr(L, "lddmm_oracle_" + nm).argtypes = [_D, _D, _D, _dbl, _int, _i64, _int, _D]
        for nm in ("applykdiff11", "applykdiff12", "applykdiff11and12"):
            getattr(L, "lddmm_oracle_" + nm).argtypes = [_D, _D, _D, _D, _dbl, _int, _i64, _int, _D]
        L.lddmm_oracle_applykmat.argtypes = [_D, _D, _D, _dbl, _int, _i64, _i64, _int, _int, _D]
        L.lddmm_oracle_applykdiffmat.argtypes = [_D, _D, _D, _dbl, _int, _i64, _i64, _int, _D]
        L.lddmm_oracle_varifold_pairs.argtypes = [_D, _D, _D, _i64, _D, _D, _D, _i64, _int, _dbl, _int, _D, _D, _D]
        L.lddmm_oracle_set_exact_coeffs.argtypes = [_int]
        L.lddmm_oracle_set_num_threads.argtypes = [_int]
        L.lddmm_oracle_num_threads.restype = _int
        _lib = L
    return _lib


def set_exact_coeffs(exact):
    """True: exact rational polynomial coefficients; False (default): the
    float32-rounded Fortran default-real literals of kernelFunctions.f90."""
    lib().lddmm_oracle_set_exact_coeffs(1 if exact else 0)


def set_num_threads(t):
    lib().lddmm_oracle_set_num_threads(int(t))


def num_threads():
    return int(lib().lddmm_oracle_num_threads())


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return a.ctypes.data_as(_D)


def _check(rc, what):
    if rc != 0:
        raise ValueError("oracle %s: unsupported kernel order for this routine" % what)


# ---- f2py-shaped entry points (kernelFunctions_fort signatures) --------------

def applyk(x, y, beta, sig, ord_):
    """kff.applyk (kernelFunctions.f90:1-54): f[k] = sum_l K(x_k, y_l) beta_l."""
    x, y, beta = _c(x), _c(y), _c(beta)
    n, d = x.shape
    m = y.shape[0]
    beta2 = beta.reshape(m, -1)
    f = np.zeros((n, beta2.shape[1]))
    _check(lib().lddmm_oracle_applyk(_p(x), _p(y), _p(beta2), float(sig), int(ord_), n, m, d, beta2.shape[1], _p(f)),
           "applyk")
    return f


def applykdifft(x, y, a1, a2, sig, ord_):
    """kff.applykdifft (kernelFunctions.f90:56-114); a1 (na,n,dimb), a2 (na,m,dimb)."""
    x, y, a1, a2 = _c(x), _c(y), _c(a1), _c(a2)
    n, d = x.shape
    m = y.shape[0]
    na, _, dimb = a1.shape
    f = np.zeros((n, d))
    _check(lib().lddmm_oracle_applykdifft(_p(x), _p(y), _p(a1), _p(a2), float(sig), int(ord_), n, m, d, dimb, na,
                                          _p(f)), "applykdifft")
    return f


def _pair_routine(nm, x, a1, a2, sig, ord_):
    x, a1, a2 = _c(x), _c(a1), _c(a2)
    n, d = x.shape
    f = np.zeros((n, d))
    _check(getattr(lib(), "lddmm_oracle_" + nm)(_p(x), _p(a1), _p(a2), float(sig), int(ord_), n, d, _p(f)), nm)
    return f


def applykdiff1(x, a1, a2, sig, ord_):
    """kff.applykdiff1 (kernelFunctions.f90:116-172)."""
    return _pair_routine("applykdiff1", x, a1, a2, sig, ord_)


def applykdiff2(x, a1, a2, sig, ord_):
    """kff.applykdiff2 (kernelFunctions.f90:174-230)."""
    return _pair_routine("applykdiff2", x, a1, a2, sig, ord_)


def applykdiff1and2(x, a1, a2, sig, ord_):
    """kff.applykdiff1and2 (kernelFunctions.f90:233-290)."""
    return _pair_routine("applykdiff1and2", x, a1, a2, sig, ord_)


def _second_routine(nm, x, a1, a2, p, sig, ord_):
    x, a1, a2, p = _c(x), _c(a1), _c(a2), _c(p)
    n, d = x.shape
    f = np.zeros((n, d))
    _check(getattr(lib(), "lddmm_oracle_" + nm)(_p(x), _p(a1), _p(a2), _p(p), float(sig), int(ord_), n, d, _p(f)),
           nm)
    return f


def applykdiff11(x, a1, a2, p, sig, ord_):
    """kff.applykdiff11 (kernelFunctions.f90:293-359), with y = x."""
    return _second_routine("applykdiff11", x, a1, a2, p, sig, ord_)


def applykdiff12(x, a1, a2, p, sig, ord_):
    """kff.applykdiff12 (kernelFunctions.f90:361-428), with y = x."""
    return _second_routine("applykdiff12", x, a1, a2, p, sig, ord_)


def applykdiff11and12(x, a1, a2, p, sig, ord_):
    """kff.applykdiff11and12 (kernelFunctions.f90:430-496)."""
    return _second_routine("applykdiff11and12", x, a1, a2, p, sig, ord_)


def applykmat(x, y, bmat, sig, ord_):
    """kff.applykmat (kernelFunctions.f90:499-552); bmat (n, m, dimb)."""
    x, y, bmat = _c(x), _c(y), _c(bmat)
    n, d = x.shape
    m = y.shape[0]
    dimb = bmat.shape[2]
    f = np.zeros((n, dimb))
    _check(lib().lddmm_oracle_applykmat(_p(x), _p(y), _p(bmat), float(sig), int(ord_), n, m, d, dimb, _p(f)),
           "applykmat")
    return f


def applykdiffmat(x, y, bmat, sig, ord_):
    """kff.applykdiffmat (kernelFunctions.f90:554-610); bmat (n, m)."""
    x, y, bmat = _c(x), _c(y), _c(bmat)
    n, d = x.shape
    m = y.shape[0]
    f = np.zeros((n, d))
    _check(lib().lddmm_oracle_applykdiffmat(_p(x), _p(y), _p(bmat), float(sig), int(ord_), n, m, d, _p(f)),
           "applykdiffmat")
    return f


def varifold_pairs(c1, n1, a1, c2, n2, a2, sig, ord_, want=("val", "z", "dz")):
    """Per-pair varifold sums (surfaces.py:1200-1254 weights formed on the fly)."""
    c1, n1, a1, c2, n2, a2 = map(_c, (c1, n1, a1, c2, n2, a2))
    nf1, d = c1.shape
    nf2 = c2.shape[0]
    val = np.zeros(nf1) if "val" in want else None
    z = np.zeros((nf1, d)) if "z" in want else None
    dz = np.zeros((nf1, d)) if "dz" in want else None
    nul = ctypes.cast(0, _D)
    rc = lib().lddmm_oracle_varifold_pairs(_p(c1), _p(n1), _p(a1), nf1, _p(c2), _p(n2), _p(a2), nf2, d, float(sig),
                                           int(ord_), _p(val) if val is not None else nul,
                                           _p(z) if z is not None else nul, _p(dz) if dz is not None else nul)
    _check(rc, "varifold_pairs")
    return val, z, dz


class FortShim:
    """Object with the f2py module ``kernelFunctions_fort`` call signatures
    (kernelFunctions.py:318-453 call sites), backed by this oracle.  Used by
    tests/golden/make_golden.py to run the reference's Python on the oracle."""

    @staticmethod
    def applyk(x, y, beta, sig, ord_, n, m, d, dimb):
        return applyk(np.asarray(x)[:n, :d], np.asarray(y)[:m, :d], np.asarray(beta).reshape(m, dimb), sig, ord_)

    @staticmethod
    def applykdifft(x, y, a1, a2, sig, ord_, n, m, d, dimb, na):
        return applykdifft(np.asarray(x)[:n, :d], np.asarray(y)[:m, :d], np.asarray(a1).reshape(na, n, dimb),
                           np.asarray(a2).reshape(na, m, dimb), sig, ord_)

    @staticmethod
    def applykmat(x, y, beta, sig, ord_, n, m, d, dimb):
        return applykmat(x, y, np.asarray(beta).reshape(n, m, dimb), sig, ord_)

    @staticmethod
    def applykdiffmat(x, y, beta, sig, ord_, n, m, d):
        return applykdiffmat(x, y, np.asarray(beta).reshape(n, m), sig, ord_)

    @staticmethod
    def applykdiff1(x, a1, a2, sig, ord_, n, d):
        return applykdiff1(x, a1, a2, sig, ord_)

    @staticmethod
    def applykdiff2(x, a1, a2, sig, ord_, n, d):
        return applykdiff2(x, a1, a2, sig, ord_)

    @staticmethod
    def applykdiff1and2(x, a1, a2, sig, ord_, n, d):
        return applykdiff1and2(x, a1, a2, sig, ord_)

    @staticmethod
    def applykdiff11and12(x, a1, a2, p, sig, ord_, n, d):
        return applykdiff11and12(x, a1, a2, p, sig, ord_)
