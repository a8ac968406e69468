"""Objective values whose precision is raised on demand.

The line search of py-lddmm's conjugateGradient.cg (conjugateGradient.py:33-217)
compares objective values with `>` / `<` and stops on |obj - objTry| < 1e-6
(absolute), and its `epsSmall` probe compares values one tiny step apart.
The objective is a small difference of norms of order |S|^2 / sigmaError^2,
so FP32c data-term sums carry errors above those thresholds near an optimum.
A _Value holds an FP32c objective value with an error bound and refines itself
to an FP64 data-term value when a comparison cannot be decided at its bound;
cg runs unchanged and takes the decisions an FP64 evaluation takes, at the
cost of FP64 sweeps for the close calls only.
"""


class _Value(float):
    """An objective value computed with FP32c data-term sums (the float value)
    with a bound on the error of DIFFERENCES of such values, that refines
    itself (prob.exact_value(ereg, x_end): an FP64 data-term value at the
    stored end point) when a comparison cannot be decided at that bound.

    Two FP32c values of one problem share most of their rounding error (same
    target cells, same packing frame, nearby geometry), so their difference is
    far more accurate than either value: a comparison is decided on the FP32c
    pair whenever |a32 - b32| exceeds the two bounds, and on the FP64 pair
    (both refined) otherwise -- never on a mixed pair, whose difference would
    carry the FP32c offset.  cg compares values with `>`, `<` and tests
    |obj - objTry| < 1e-6; these operators (and their reflections, which
    Python tries first for a float subclass) implement that rule, so every
    decision is the one an FP64 evaluation takes as long as the bound holds.
    Each double refinement measures the actual difference error and raises
    the problem's bound (prob.noise_obs, see value_bound) when it was larger."""

    def __new__(cls, value, prob=None, ereg=0.0, x_end=None, err=0.0):
        o = float.__new__(cls, value)
        o.v32 = float(value)
        o.best = float(value)
        o.prob = prob
        o.ereg = ereg
        o.x_end = x_end
        o.err = float(err)
        o.exact = not (err > 0.0)
        return o

    def refine(self):
        if not self.exact:
            self.best = self.prob.exact_value(self.ereg, self.x_end)
            self.exact = True
            self.x_end = None
        return self.best


def _resolve(a, b, margin=0.0):
    """a - b, decided as described in _Value (margin: a threshold the caller
    compares |a - b| with, the 1e-6 of the stop test)."""
    va, vb = isinstance(a, _Value), isinstance(b, _Value)
    if va and vb:
        if a.exact and b.exact:
            return a.best - b.best
        d32 = a.v32 - b.v32
        if abs(d32) > a.err + b.err + margin:
            return d32
        a.refine()
        b.refine()
        d64 = a.best - b.best
        obs = abs(d32 - d64)
        for v in (a, b):
            if v.prob is not None:
                v.prob.noise_obs = max(getattr(v.prob, "noise_obs", 0.0), obs)
        return d64
    if not va and not vb:
        return float(a) - float(b)
    # one plain float: compare with the exact value unless the gap is huge
    v, x, sign = (a, float(b), 1.0) if va else (b, float(a), -1.0)
    d = sign * (v.best - x)
    if v.exact or abs(d) > 100.0 * v.err + margin:
        return d
    v.refine()
    return sign * (v.best - x)


def _gt(a, b):
    return _resolve(a, b) > 0


def _lt(a, b):
    return _resolve(a, b) < 0


def _ge(a, b):
    return _resolve(a, b) >= 0


def _le(a, b):
    return _resolve(a, b) <= 0


def _sub(a, b):
    return _resolve(a, b, margin=1e-6)


def _rsub(a, b):
    return _resolve(b, a, margin=1e-6)


_Value.__gt__ = _gt
_Value.__lt__ = _lt
_Value.__ge__ = _ge
_Value.__le__ = _le
_Value.__sub__ = _sub
_Value.__rsub__ = _rsub
_Value.__hash__ = float.__hash__


def value_bound(prob, noise, scale):
    """Difference-error bound of a new value: noise x |scale|, raised to twice
    the largest difference error measured so far on this problem."""
    return max(noise * abs(scale), 2.0 * getattr(prob, "noise_obs", 0.0))
