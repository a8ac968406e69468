"""conjugateGradient.cg on the host, against the oracle's restatement.

The optimiser only compares host scalars, so a mock problem (a 2-D quadratic
whose gradient is wrong once) drives it through the "bad direction" branch of
py-lddmm/conjugateGradient.py:143-154.  There the reference disables CG and
skips the update only under ``if verb:``; with verb false it falls through to
the halving / growth loops and accepts the trial.  Both behaviours are kept.
"""
import logging

import numpy as np
import pytest

from oracle import lddmm_ref as ref
from registration_b200 import conjugateGradient as cgp


class _Quadratic:
    """f(x) = |A x|^2; the gradient of iteration `lie_at` is rotated by
    `angle` degrees and scaled, so that PR+ keeps beta > 0 and the direction
    goes uphill.  updateTry keeps the trial only when it improves on objRef,
    as SurfaceMatching.updateTry does (surfaceMatching.py:255-289)."""

    def __init__(self, lie_at=1, angle=150.0, scale=5.0):
        self.x = np.array([1.0, 0.7])
        self.A = np.diag([1.0, 3.0])
        th = np.deg2rad(angle)
        self.R = scale * np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
        self.lie_at, self.calls, self.accepted, self.trials = lie_at, 0, [], []
        self.xtry = None

    def _f(self, x):
        return float(np.sum((self.A @ x) ** 2))

    def getVariable(self):
        return self.x

    def objectiveFun(self):
        return self._f(self.x)

    def getGradient(self, coeff):
        g = 2.0 * self.A.T @ self.A @ self.x
        if self.calls == self.lie_at:
            g = self.R @ g
        self.calls += 1
        return g

    def updateTry(self, d, eps, objRef=None):
        xt = self.x - eps * d
        v = self._f(xt)
        self.trials.append((float(eps), v))
        if objRef is None or v < objRef:
            self.xtry = xt
        return v

    def acceptVarTry(self):
        self.x = self.xtry.copy()
        self.accepted.append(self.calls)

    def dotProduct(self, g, gs):
        return [float(g @ h) for h in gs]

    def copyDir(self, g):
        return np.copy(g)

    def addProd(self, a, b, c):
        return a + c * b

    def randomDir(self):
        return np.ones(2)


@pytest.mark.parametrize("verb", [True, False])
def test_bad_direction_branch_follows_the_reference(verb, caplog):
    a, b = _Quadratic(), _Quadratic()
    with caplog.at_level(logging.INFO):
        cgp.cg(a, verb=verb, maxIter=4, epsInit=0.1)
    ref.cg(b, verb=verb, maxIter=4, epsInit=0.1)
    assert a.trials == b.trials and a.accepted == b.accepted
    np.testing.assert_array_equal(a.x, b.x)
    if verb:
        # CG disabled, no update in the iteration with the lying gradient
        assert "Disabling CG: bad direction" in caplog.text
        assert a.accepted == [1, 3, 4]
    else:
        # the reference goes on with the line search and accepts
        assert "Disabling CG" not in caplog.text
        assert a.accepted == [1, 2, 3, 4]
