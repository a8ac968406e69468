"""Host logic of the batched trial steps (registration_b200/_matching.py), no
GPU: the step-size ladders are the values cg computes (the same floating-point
operations), hold the tiny-step probe, and have the batch size; the best trial's
state is copied out of its batch slot only when read or accepted; and on the
step sizes of a recorded line search the batches answer every trial."""
import numpy as np
import pytest
import torch

from registration_b200 import _matching as M
from registration_b200 import conjugateGradient as CG


def _bare(B):
    m = M.DeviceMatching.__new__(M.DeviceMatching)
    m._graph = {"B": B}
    return m


def _halvings(e, k):
    out = [e]
    for _ in range(k - 1):
        out.append(out[-1] / 2)
    return out


@pytest.mark.parametrize("B", [1, 8, 16, 24])
def test_ladders(B):
    m = _bare(B)
    d = object()
    eps0, probe = 0.37, 3.1e-7
    m._hint = (d, [eps0, probe])
    lad = m._trial_ladder(eps0, {}, d)
    assert len(lad) == B and len(set(lad)) == B and lad[0] == eps0
    if B == 1:
        return
    h = _halvings(eps0, min(12, B - 1))
    assert lad[:len(h)] == h                              # eps / 2 chained, as cg's eps = eps / 2
    assert probe in lad
    if B >= 24:                                           # first two growth steps of halving depth 5
        g1 = 1.25 * h[5]
        assert g1 in lad and 1.25 * g1 in lad
    # a growth step of an evaluated size gets the growth chain, as cg's eps *= 1.25
    e_f = h[6]
    grow = m._trial_ladder(1.25 * e_f, set(lad), d)
    want = [1.25 * e_f]
    while len(want) < B:
        want.append(1.25 * want[-1])
    assert grow == want
    # another direction: its hint does not apply
    lad2 = m._trial_ladder(eps0, {}, object())
    assert probe not in lad2 and len(lad2) == B


class _Recorder:
    """A quadratic objective driven by the product cg that records the step
    sizes of every updateTry call, with the batched path's answer rule: a call
    is served by the last batch when its step size is in it, else a new batch
    is formed by _trial_ladder."""

    def __init__(self, B):
        self.m = _bare(B)
        self.x = np.array([3.0, -2.0, 1.5])
        self.A = np.diag([1.0, 10.0, 100.0])
        self.batches = 0
        self.calls = 0
        self.cache = set()
        self.dir_id = None
        self.obj = None

    def getVariable(self):
        return self.x

    def _f(self, x):
        return 0.5 * float(x @ self.A @ x)

    def objectiveFun(self):
        self.obj = self._f(self.x)
        return self.obj

    def expectTrials(self, dir, steps):
        self.m._hint = (dir, [float(e) for e in steps])

    def updateTry(self, dir, eps, objRef=None):
        self.calls += 1
        if self.dir_id is not dir:
            self.dir_id, self.cache = dir, set()
        if eps not in self.cache:
            self.batches += 1
            self.cache = set(self.m._trial_ladder(float(eps), self.cache, dir))
            assert eps in self.cache
        xt = self.x - eps * dir
        v = self._f(xt)
        if objRef is None or v < objRef:
            self.xtry, self.objTry = xt, v
        return v

    def acceptVarTry(self):
        self.x = self.xtry
        self.obj = self.objTry

    def getGradient(self, coeff=1.0):
        return self.A @ self.x / coeff


def test_batches_answer_a_cg_line_search():
    # the same cg decisions with one-step-size batches and with 24-step batches
    traces = {}
    for B in (1, 24):
        r = _Recorder(B)
        CG.cg(r, verb=False, maxIter=30, epsInit=1.0)
        traces[B] = (r.x.copy(), r.calls, r.batches)
    (x1, c1, b1), (x24, c24, b24) = traces[1], traces[24]
    assert np.array_equal(x1, x24) and c1 == c24
    assert b1 == c1 and b24 < c24 / 2, (b24, c24)


def test_best_trial_copied_out_of_its_slot_only_when_needed():
    m = M.DeviceMatching.__new__(M.DeviceMatching)
    g = {"atTry": torch.arange(24.0).reshape(3, 2, 4), "xt": torch.arange(30.0).reshape(3, 10)}
    m.atTry = torch.zeros(2, 4)
    m._pending_try = (g, 1)
    m.objTry = 5.0
    got = m.atTry                                        # read: copied out now
    assert torch.equal(got, g["atTry"][1]) and got.data_ptr() != g["atTry"][1].data_ptr()
    assert m._pending_try is None and torch.equal(m.xtTry, g["xt"][1])
    # accepted straight from the slot
    m._pending_try = (g, 2)
    m.acceptVarTry()
    assert m.obj == 5.0 and torch.equal(m.at, g["atTry"][2]) and torch.equal(m.xt, g["xt"][2])
    g["atTry"][2].fill_(-1.0)                            # the slot is reused by the next batch
    assert torch.equal(m.at, torch.arange(16.0, 24.0).reshape(2, 4))


def test_ladders_are_distinct_and_full():
    """A batch's step sizes are distinct (they key the batch's values) and fill it."""
    rng = np.random.default_rng(0)
    d = object()
    for B in (1, 2, 3, 5, 8, 13, 16, 20, 24, 32):
        m = _bare(B)
        for _ in range(200):
            e, p = float(10 ** rng.uniform(-8, 3)), float(10 ** rng.uniform(-9, -5))
            m._hint = (d, [e, p])
            lad = m._trial_ladder(e, {}, d)
            assert len(lad) == B and len(set(lad)) == B
            grow = m._trial_ladder(1.25 * lad[min(3, B - 1)], set(lad), d)
            assert len(grow) == B and len(set(grow)) == B


def test_cg_hints_the_probe_it_then_tries():
    """cg's optional hint names, before each line search, the first step size
    and the tiny-step probe; when the first trial fails, the probe cg tries is
    exactly the hinted value (so a batch holding it answers the call)."""

    class Hinted(_Recorder):
        def __init__(self):
            super().__init__(1)
            self.hints, self.first = [], []

        def expectTrials(self, dir, steps):
            self.hints.append((dir, list(steps)))

        def updateTry(self, dir, eps, objRef=None):
            if self.hints and self.hints[-1][0] is dir:
                self.first.append((len(self.hints), float(eps)))
            return super().updateTry(dir, eps, objRef)

    r = Hinted()
    r.x = np.array([30.0, -20.0, 15.0])      # far from the optimum: the first steps overshoot
    CG.cg(r, verb=False, maxIter=15, epsInit=10.0)
    assert r.hints
    probes = 0
    for i, (d, steps) in enumerate(r.hints, start=1):
        tried = [e for k, e in r.first if k == i]
        assert tried and tried[0] == steps[0]          # the first trial is the hinted step
        if len(tried) > 1 and tried[1] < steps[0] / 1000:
            assert tried[1] == steps[1]                # the probe is the hinted value
            probes += 1
    assert probes >= 1
