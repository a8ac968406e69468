"""ctypes binding of liblddmm_b200.so (the C ABI declared in include/lddmm_b200.h).

The shared library is built in-tree by ``python -m registration_b200.build``.
There is no CPU fallback: if the library or a CUDA device is missing, every
operation raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblddmm_b200.so")

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I = ctypes.c_int
_D = ctypes.c_double
_SZ = ctypes.c_size_t

# name -> (restype, argtypes); mirrors include/lddmm_b200.h
SIGNATURES = {
    "lddmm_last_error": (ctypes.c_char_p, []),
    "lddmm_abi_version": (_I, []),
    "lddmm_applyk_f32c_workspace": (_SZ, [_I64, _I64, _I, _I]),
    "lddmm_applyk_f64_workspace": (_SZ, [_I64, _I64, _I, _I]),
    "lddmm_applyk_f32c": (_I, [_P, _I64, _P, _I64, _P, _I, _I, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applyk_f64": (_I, [_P, _I64, _P, _I64, _P, _I, _I, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applyk_f32c_noalloc": (_I, [_P, _I64, _P, _I64, _P, _I, _I, _D, _I, _P, _P]),
    "lddmm_applykdifft_f32c_workspace": (_SZ, [_I64, _I64, _I, _I, _I]),
    "lddmm_applykdifft_f64_workspace": (_SZ, [_I64, _I64, _I, _I, _I]),
    "lddmm_applykdifft_f32c": (_I, [_P, _I64, _P, _I64, _P, _P, _I, _I, _I, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdifft_f64": (_I, [_P, _I64, _P, _I64, _P, _P, _I, _I, _I, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_moments_f64_workspace": (_SZ, [_I64, _I, _I]),
    "lddmm_moments_f64": (_I, [_P, _I64, _I, _P, _I, _P, _P, _P, _SZ, _P]),
    "lddmm_rows_affine_f64": (_I, [_P, _I64, _I, _P, _P, _P, _I, _P, _P]),
    "lddmm_applydiv_f32c_workspace": (_SZ, [_I64, _I64, _I]),
    "lddmm_applydiv_f64_workspace": (_SZ, [_I64, _I64, _I]),
    "lddmm_applydiv_f32c": (_I, [_P, _I64, _P, _I64, _P, _I, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applydiv_f64": (_I, [_P, _I64, _P, _I64, _P, _I, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_shoot_f32c_workspace": (_SZ, [_I64, _I, _I]),
    "lddmm_shoot_f64_workspace": (_SZ, [_I64, _I, _I]),
    "lddmm_shoot_f32c": (_I, [_P, _I64, _I, _P, _I, _D, _D, _I, _D, _P, _P, _P, _SZ, _P]),
    "lddmm_shoot_f64": (_I, [_P, _I64, _I, _P, _I, _D, _D, _I, _D, _P, _P, _P, _SZ, _P]),
    "lddmm_shoot_along_f32c": (_I, [_P, _I64, _I, _P, _P, _P, _I, _D, _D, _I, _D, _P, _P, _P, _P, _SZ, _P]),
    "lddmm_shoot_along_f64": (_I, [_P, _I64, _I, _P, _P, _P, _I, _D, _D, _I, _D, _P, _P, _P, _P, _SZ, _P]),
    "lddmm_shoot_along_batch_f32c_workspace": (_SZ, [_I64, _I, _I, _I]),
    "lddmm_shoot_along_batch_f64_workspace": (_SZ, [_I64, _I, _I, _I]),
    "lddmm_shoot_along_batch_f32c": (_I, [_P, _I64, _I, _P, _P, _P, _I, _I, _D, _D, _I, _D, _P, _P, _P, _P, _SZ,
                                          _P]),
    "lddmm_shoot_along_batch_f64": (_I, [_P, _I64, _I, _P, _P, _P, _I, _I, _D, _D, _I, _D, _P, _P, _P, _P, _SZ,
                                         _P]),
    "lddmm_trial_batch_size": (_I, [_I64, _I, _I64, _I64, _I, _I]),
    "lddmm_metric_dots_f32c_workspace": (_SZ, [_I64, _I, _I, _I]),
    "lddmm_metric_dots_f64_workspace": (_SZ, [_I64, _I, _I, _I]),
    "lddmm_metric_dots_f32c": (_I, [_P, _I64, _I, _I, _P, _P, _I, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_metric_dots_f64": (_I, [_P, _I64, _I, _I, _P, _P, _I, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_covector_f32c_workspace": (_SZ, [_I64, _I, _I]),
    "lddmm_covector_f64_workspace": (_SZ, [_I64, _I, _I]),
    "lddmm_covector_f32c": (_I, [_P, _I64, _I, _P, _I, _D, _P, _D, _I, _D, _P, _P, _P, _SZ, _P]),
    "lddmm_covector_f64": (_I, [_P, _I64, _I, _P, _I, _D, _P, _D, _I, _D, _P, _P, _P, _SZ, _P]),
    "lddmm_dataterm_f32c_workspace": (_SZ, [_I, _I, _I64, _I, _I64, _I64, _I, _I, _I]),
    "lddmm_dataterm_f64_workspace": (_SZ, [_I, _I, _I64, _I, _I64, _I64, _I, _I, _I]),
    "lddmm_dataterm_f32c": (_I, [_I, _I, _P, _I64, _I, _P, _I64, _P, _P, _I64, _D, _I, _D, _D, _P, _P, _P, _P,
                                 _P, _SZ, _P]),
    "lddmm_dataterm_f64": (_I, [_I, _I, _P, _I64, _I, _P, _I64, _P, _P, _I64, _D, _I, _D, _D, _P, _P, _P, _P,
                                _P, _SZ, _P]),
    "lddmm_dataterm_value_batch_f32c_workspace": (_SZ, [_I, _I, _I64, _I, _I64, _I64, _I, _I]),
    "lddmm_dataterm_value_batch_f64_workspace": (_SZ, [_I, _I, _I64, _I, _I64, _I64, _I, _I]),
    "lddmm_dataterm_value_batch_f32c": (_I, [_I, _I, _P, _I64, _I, _P, _I64, _P, _P, _I64, _D, _I, _D, _D, _I, _I64,
                                             _P, _P, _SZ, _P]),
    "lddmm_dataterm_value_batch_f64": (_I, [_I, _I, _P, _I64, _I, _P, _I64, _P, _P, _I64, _D, _I, _D, _D, _I, _I64,
                                            _P, _P, _SZ, _P]),
    "lddmm_epdiff_f32c_workspace": (_SZ, [_I64, _I, _I]),
    "lddmm_epdiff_f64_workspace": (_SZ, [_I64, _I, _I]),
    "lddmm_epdiff_f32c": (_I, [_P, _I64, _I, _P, _I, _D, _I, _P, _P, _P, _SZ, _P]),
    "lddmm_epdiff_f64": (_I, [_P, _I64, _I, _P, _I, _D, _I, _P, _P, _P, _SZ, _P]),
    "lddmm_applykmat_f32c": (_I, [_P, _I64, _P, _I64, _P, _I, _I, _D, _I, _P, _P]),
    "lddmm_applykmat_f64": (_I, [_P, _I64, _P, _I64, _P, _I, _I, _D, _I, _P, _P]),
    "lddmm_applykdiffmat_f32c": (_I, [_P, _I64, _P, _I64, _P, _I, _D, _I, _P, _P]),
    "lddmm_applykdiffmat_f64": (_I, [_P, _I64, _P, _I64, _P, _I, _D, _I, _P, _P]),
    "lddmm_applykdiffx_f32c_workspace": (_SZ, [_I, _I64, _I, _I]),
    "lddmm_applykdiffx_f64_workspace": (_SZ, [_I, _I64, _I, _I]),
    "lddmm_applykdiff1_f32c": (_I, [_P, _I64, _I, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff1_f64": (_I, [_P, _I64, _I, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff2_f32c": (_I, [_P, _I64, _I, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff2_f64": (_I, [_P, _I64, _I, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff1and2_f32c": (_I, [_P, _I64, _I, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff1and2_f64": (_I, [_P, _I64, _I, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff11_f32c": (_I, [_P, _I64, _I, _P, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff11_f64": (_I, [_P, _I64, _I, _P, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff12_f32c": (_I, [_P, _I64, _I, _P, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff12_f64": (_I, [_P, _I64, _I, _P, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff11and12_f32c": (_I, [_P, _I64, _I, _P, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    "lddmm_applykdiff11and12_f64": (_I, [_P, _I64, _I, _P, _P, _P, _D, _I, _P, _P, _SZ, _P]),
    # ragged launches: offset / sigma / regweight arguments are host arrays
    "lddmm_ragged_shoot_f32c_workspace": (_SZ, [_I, _P, _I, _I, _I]),
    "lddmm_ragged_shoot_f32c": (_I, [_I, _P, _I, _P, _P, _I, _P, _I, _P, _P, _P, _P, _SZ, _P]),
    "lddmm_ragged_covector_f32c_workspace": (_SZ, [_I, _P, _I, _I, _I]),
    "lddmm_ragged_covector_f32c": (_I, [_I, _P, _I, _P, _P, _I, _P, _P, _I, _P, _P, _P, _P, _SZ, _P]),
    "lddmm_ragged_applyk_f32c_workspace": (_SZ, [_I, _P, _P, _I, _I, _I]),
    "lddmm_ragged_applyk_f32c": (_I, [_I, _P, _P, _P, _P, _I, _P, _P, _P, _I, _P, _I, _P, _P, _SZ, _P]),
    "lddmm_ragged_dataterm_f32c_workspace": (_SZ, [_I, _I, _I, _P, _P, _P, _I, _I, _I, _I]),
    "lddmm_ragged_dataterm_f64_workspace": (_SZ, [_I, _I, _I, _P, _P, _P, _I, _I, _I, _I]),
    "lddmm_ragged_dataterm_f32c": (_I, [_I, _I, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P, _I, _D, _D, _P, _P, _P, _P,
                                        _P, _P, _SZ, _P]),
    "lddmm_ragged_dataterm_f64": (_I, [_I, _I, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P, _I, _D, _D, _P, _P, _P, _P,
                                       _P, _P, _SZ, _P]),
}

ERRORS = {-1: "invalid argument", -2: "workspace too small", -3: "CUDA error", -4: "unsupported"}

_lib = None


class LddmmError(RuntimeError):
    pass


def load():
    """Loads the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LddmmError("liblddmm_b200.so not found at %s; build it with "
                             "`python -m registration_b200.build` (no CPU fallback exists)" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def call(name, *args):
    rc = getattr(load(), name)(*args)
    if rc != 0:
        msg = load().lddmm_last_error().decode(errors="replace")
        kind = ERRORS.get(rc, "error %d" % rc)
        if rc == -1:
            raise ValueError("%s: %s (%s)" % (name, msg, kind))
        raise LddmmError("%s: %s (%s)" % (name, msg, kind))
    return rc


def query(name, *args):
    return int(getattr(load(), name)(*args))
