"""Host logic of the continuous-batching scheduler (no GPU): admission under
the slot count and the HBM budget, late arrivals, grouping of work into one
launch per kind, error isolation and result routing.  The work items are
computed by a numpy stand-in engine (quadratic objectives), so every request's
answer is known in closed form."""
import threading
import time

import numpy as np
import pytest

from registration_b200 import serving


class _Dir:
    def __init__(self, diff):
        self.diff = diff


class _ToyProblem:
    """E(a) = sum w (a - c)^2 + 1; the cg protocol with every evaluation posted."""

    def __init__(self, req, eng):
        self.req, self.engine = req, eng
        self.at = np.zeros(req.n)
        self.atTry = self.at
        self.xt = None
        self.obj = self.objTry = None
        self.gradCoeff = 1.0
        self.iters = 0
        self.converged = False
        self.calls = {"value": 0, "grad": 0, "dot": 0}

    def getVariable(self):
        return [self.at]

    def objectiveFun(self):
        if self.obj is None:
            self.obj = self.engine.post(self, "value", self.at)
        return self.obj

    def updateTry(self, dir, eps, objRef=None):
        a = self.at - eps * dir.diff
        e = self.engine.post(self, "value", a)
        if objRef is None or e < objRef:
            self.atTry, self.objTry = a, e
        return e

    def getGradient(self, coeff=1.0):
        return _Dir(self.engine.post(self, "grad", self.at) / coeff)

    def dotProduct(self, g1, g2):
        return self.engine.post(self, "dot", (g1.diff, [g.diff for g in g2]))

    def addProd(self, d1, d2, beta):
        return _Dir(d1.diff + beta * d2.diff)

    def copyDir(self, d0):
        return _Dir(d0.diff.copy())

    def acceptVarTry(self):
        self.at, self.obj = self.atTry, self.objTry

    def endOfIteration(self):
        self.iters += 1


class _ToyRequest:
    def __init__(self, rid, n, group=0, fail=False, max_iter=30):
        rng = np.random.default_rng(rid)
        self.rid, self.n, self.group, self.fail = rid, n, group, fail
        self.w = rng.uniform(0.5, 2.0, n)
        self.c = rng.standard_normal(n)
        self.max_iter = max_iter
        self.arrival = self.start = self.finish = None
        self.result = self.error = None
        self.done = threading.Event()

    def hbm_bytes(self):
        return 1000 * self.n

    def latency(self):
        return self.finish - self.arrival


class _ToyEngine(serving.Scheduler):
    def __init__(self, **kw):
        super().__init__(**kw)
        self.launch_log = []
        self.lock = threading.Lock()

    def _make_problem(self, req):
        return _ToyProblem(req, self)

    def _log(self, kind, items):
        self.launch_log.append((kind, sorted(p.req.rid for p, _ in items), len({p.req.group for p, _ in items})))

    def _do_value(self, items):
        self._log("value", items)
        out = []
        for p, a in items:
            if p.req.fail:
                raise RuntimeError("planted failure")
            out.append(float((p.req.w * (a - p.req.c) ** 2).sum() + 1.0))
            p.calls["value"] += 1
        return out

    def _do_grad(self, items):
        self._log("grad", items)
        return [2 * p.req.w * (a - p.req.c) for p, a in items]

    def _do_dot(self, items):
        self._log("dot", items)
        return [np.array([float((g1 * g).sum()) for g in g2s]) for p, (g1, g2s) in items]


def _alone(req):
    eng = _ToyEngine()
    r = _ToyRequest(req.rid, req.n, req.group, req.fail, req.max_iter)
    eng.submit(r)
    eng.run()
    return r


def test_all_requests_finish_and_match_alone():
    reqs = [_ToyRequest(i, 5 + 3 * i) for i in range(8)]
    eng = _ToyEngine(max_active=8)
    for r in reqs:
        eng.submit(r)
    eng.run()
    st = eng.stats()
    assert st["finished"] == 8 and st["failed"] == 0 and st["max_batch"] == 8
    for r in reqs:
        a = _alone(r)
        assert r.result["obj"] == a.result["obj"] and np.array_equal(r.result["at"], a.result["at"])
        # the minimiser of the quadratic is c, E = 1
        assert abs(r.result["obj"] - 1.0) < 1e-6


def test_slot_count_and_budget_limit_admission():
    reqs = [_ToyRequest(i, 10) for i in range(6)]
    eng = _ToyEngine(max_active=3)
    for r in reqs:
        eng.submit(r)
    eng.run()
    assert eng.stats()["max_active"] == 3
    assert max(len(rids) for _, rids, _ in eng.launch_log) <= 3
    reqs = [_ToyRequest(i, 10) for i in range(6)]
    eng = _ToyEngine(hbm_budget_bytes=2 * 10 * 1000 + 1)     # two requests' state
    for r in reqs:
        eng.submit(r)
    eng.run()
    assert eng.stats()["max_active"] == 2 and eng.stats()["finished"] == 6


def test_request_above_budget_is_rejected_others_served():
    big, small = _ToyRequest(0, 100), _ToyRequest(1, 5)
    eng = _ToyEngine(hbm_budget_bytes=50 * 1000)
    eng.submit(big)
    eng.submit(small)
    eng.run()
    assert isinstance(big.error, MemoryError) and small.error is None


def test_late_arrivals_join_running_batches():
    reqs = [_ToyRequest(i, 8, max_iter=200) for i in range(4)]
    t0 = time.perf_counter()
    eng = _ToyEngine()
    for j, r in enumerate(reqs):
        eng.submit(r, arrival=t0 + 0.02 * j)
    eng.run()
    for r in reqs:
        assert r.start >= r.arrival and r.error is None
        a = _alone(r)
        assert r.result["obj"] == a.result["obj"]


def test_groups_never_share_a_launch_and_failures_are_isolated():
    reqs = [_ToyRequest(0, 6, group=0), _ToyRequest(1, 7, group=1), _ToyRequest(2, 8, group=0),
            _ToyRequest(3, 9, group=1, fail=True)]
    eng = _ToyEngine()
    for r in reqs:
        eng.submit(r)
    eng.run()
    assert all(ngroups == 1 for _, _, ngroups in eng.launch_log)
    assert isinstance(reqs[3].error, RuntimeError)
    for r in reqs[:3]:
        assert r.error is None and r.result["obj"] == _alone(r).result["obj"]


def test_lanes_split_rounds_by_size_and_keep_results():
    reqs = [_ToyRequest(i, n) for i, n in enumerate([4, 40, 5, 60, 6, 80])]
    eng = _ToyEngine(lanes=(10, 50))
    for r in reqs:
        eng.submit(r)
    eng.run()
    st = eng.stats()
    assert st["failed"] == 0 and all(n > 0 for n in st["lane_rounds"])
    bounds = [10, 50, float("inf")]
    for kind, rids, _ in eng.launch_log:
        lanes = {next(k for k, b in enumerate(bounds) if reqs[i].n <= b) for i in rids}
        assert len(lanes) == 1          # a launch never mixes lanes
    for r in reqs:
        assert r.result["obj"] == _alone(r).result["obj"]


def test_latency_percentiles_reported():
    reqs = [_ToyRequest(i, 4) for i in range(5)]
    eng = _ToyEngine()
    for r in reqs:
        eng.submit(r)
    eng.run()
    st = eng.stats()
    assert 0 < st["p50_s"] <= st["p99_s"]


class _FakeProb:
    def __init__(self, exact):
        self.exact = exact
        self.refines = 0

    def exact_value(self, ereg, x_end):
        self.refines += 1
        return self.exact[x_end]


def test_values_refine_only_when_the_bound_cannot_decide():
    from registration_b200._precision import _Value as V
    # FP32c values carry a common offset (+0.0003) that cancels in differences
    p = _FakeProb({"a": 10.0001, "b": 10.0, "c": 12.0, "d": 10.0000005})
    a = V(10.0004, p, 0.0, "a", 1e-3)
    b = V(10.0003, p, 0.0, "b", 1e-3)
    c = V(12.0003, p, 0.0, "c", 1e-3)
    assert c > b and b < c and p.refines == 0          # |a32 - b32| > bounds: FP32c decides
    assert a > b and p.refines == 2                     # within bounds: both refined, exact 10.0001 > 10.0
    assert a.best == 10.0001 and a.exact and p.noise_obs < 1e-12
    # a refined value against an unrefined one is compared on the FP32c pair
    e = V(10.0053, p, 0.0, "c", 1e-3)
    assert e > a and p.refines == 2
    d = V(10.0003005, p, 0.0, "d", 1e-3)
    # |obj - objTry| < 1e-6 test: refined to the exact 5e-7 difference
    assert abs(d - b) < 1e-6 and p.refines == 3
    assert 12.5 > c and c < 12.5 and float(c) == 12.0003   # plain floats on either side
    assert 1e500 > a


def test_value_bound_grows_with_measured_error():
    from registration_b200._precision import _Value as V, value_bound
    p = _FakeProb({"a": 1.0, "b": 2.0})
    assert value_bound(p, 1e-8, 100.0) == 1e-6
    a, b = V(1.0 + 3e-7, p, 0.0, "a", 1e-6), V(1.0 + 4e-7, p, 0.0, "b", 1e-6)
    assert a < b            # undecided at the bound: refined, exact 1.0 < 2.0
    assert abs(p.noise_obs - (1.0 - 1e-7)) < 1e-12
    assert value_bound(p, 1e-8, 100.0) == 2 * p.noise_obs


@pytest.mark.parametrize("bad", ["errorType"])
def test_match_request_validation(bad):
    class P:
        timeStep = 0.1
        errorType = "hausdorff"
    with pytest.raises(ValueError):
        serving.MatchRequest(None, None, P())


def test_match_request_orients_target_and_picks_the_protocol_step():
    """A surface target with the opposite orientation gets its faces flipped, as
    SurfaceMatching does (surfaceMatching.py:126-129); curves keep cg's default
    first step (epsInit 10, curveMatching.py:352), surfaces use 0.1."""
    from registration_b200 import curves as cv
    from registration_b200 import geometry as geo
    from registration_b200 import surfaces as sf

    class P:
        timeStep = 0.2
        errorType = "current"
    v, f = geo.icosphere(1)
    inward = f[:, [0, 2, 1]]
    r = serving.MatchRequest(sf.Surface(FV=[f, v]), sf.Surface(FV=[inward, 1.1 * v]), P())
    np.testing.assert_array_equal(r.f1, f)
    assert r.eps_init == 0.1
    same = serving.MatchRequest(sf.Surface(FV=[f, v]), sf.Surface(FV=[f, 1.1 * v]), P())
    np.testing.assert_array_equal(same.f1, f)
    c, _ = geo.ellipse_curve(32)
    rc = serving.MatchRequest(cv.Curve(pointSet=c), cv.Curve(pointSet=1.1 * c), P())
    assert rc.f0.shape[1] == 2 and rc.eps_init == 10.0


class _CancellingEngine(_ToyEngine):
    """Cancels request `victim` once it has taken `after` value launches."""

    def __init__(self, victim, after, **kw):
        super().__init__(**kw)
        self.victim, self.after = victim, after

    def _do_value(self, items):
        for p, _ in items:
            if p.req is self.victim and p.calls["value"] >= self.after:
                self.victim.cancelled = True
        return super()._do_value(items)


def test_cancelled_requests_end_and_free_their_slot():
    """A queued request cancelled before admission never starts; an active one
    stops at its next GPU call.  Both end with RequestCancelled, give back their
    slot and budget, and the others finish exactly as alone."""
    reqs = [_ToyRequest(i, 6 + i, max_iter=60) for i in range(4)]
    queued = _ToyRequest(9, 5)
    queued.cancelled = True
    eng = _CancellingEngine(reqs[1], after=3, max_active=4)
    for r in reqs + [queued]:
        eng.submit(r)
    eng.run()
    assert isinstance(queued.error, serving.RequestCancelled) and queued.start == queued.finish
    assert isinstance(reqs[1].error, serving.RequestCancelled)
    assert eng.n_active == 0 and eng.hbm_in_use == 0 and not eng.threads
    assert eng.stats()["failed"] == 2
    for r in (reqs[0], reqs[2], reqs[3]):
        assert r.error is None and r.result["obj"] == _alone(r).result["obj"]


class _BadInput(_ToyRequest):
    def input_error(self):
        return ValueError("request %s: target vertices are not finite" % self.rid)


def test_invalid_inputs_fail_at_admission_others_served():
    bad, good = _BadInput(0, 5), _ToyRequest(1, 7)
    eng = _ToyEngine()
    eng.submit(bad)
    eng.submit(good)
    eng.run()
    assert isinstance(bad.error, ValueError) and bad.result is None
    assert good.error is None and good.result["obj"] == _alone(good).result["obj"]


class _InterruptedEngine(_ToyEngine):
    """run() leaves on an exception while requests are waiting for rounds."""

    def __init__(self, **kw):
        super().__init__(**kw)
        self.values = 0

    def _do_value(self, items):
        self.values += 1
        return super()._do_value(items)

    def _can_admit(self, now):
        if self.values >= 4:
            raise KeyboardInterrupt
        return super()._can_admit(now)


def test_run_leaving_on_an_exception_ends_every_request_thread():
    reqs = [_ToyRequest(i, 6, max_iter=500) for i in range(3)]
    late = _ToyRequest(7, 6)
    eng = _InterruptedEngine()
    for r in reqs:
        eng.submit(r)
    eng.submit(late, arrival=time.perf_counter() + 3600.0)
    done = threading.Event()
    caught = []

    def drive():
        try:
            eng.run()
        except KeyboardInterrupt as exc:
            caught.append(exc)
        done.set()

    th = threading.Thread(target=drive, daemon=True)
    th.start()
    assert done.wait(30.0), "run() did not return: request threads were left blocked"
    assert caught and not eng.threads
    for r in reqs + [late]:
        assert r.done.is_set() and r.error is not None
    assert isinstance(late.error, serving.ServingStopped)


def test_match_request_input_checks():
    from registration_b200 import geometry as geo
    from registration_b200 import surfaces as sf

    class P:
        timeStep = 0.2
        errorType = "varifold"
    v, f = geo.icosphere(1)
    ok = serving.MatchRequest(sf.Surface(FV=[f, v]), sf.Surface(FV=[f, 1.1 * v]), P())
    assert ok.input_error() is None
    vt = 1.1 * v
    vt[3, 1] = np.nan
    assert "target vertices" in str(serving.MatchRequest(sf.Surface(FV=[f, v]), sf.Surface(FV=[f, vt]),
                                                         P()).input_error())
    at = np.zeros((5, len(v), 3))
    at[2, 0, 0] = np.inf
    r = serving.MatchRequest(sf.Surface(FV=[f, v]), sf.Surface(FV=[f, 1.1 * v]), P(), at_init=at)
    assert "initial momenta" in str(r.input_error())
    with pytest.raises(ValueError):
        serving.MatchRequest(sf.Surface(FV=[f, v]), sf.Surface(FV=[f, 1.1 * v]), P(), at_init=at[:2])
