"""Continuous-batching server for surface / curve matching requests.

Each request is a matching problem with the interface of
py-lddmm/surfaceMatching.py:74-484 (or curveMatching.py:58-354): Euler
shooting of the template, a current / measure / varifold data term and the
conjugate-gradient loop of conjugateGradient.cg.  The optimiser of every
request runs unchanged in its own host thread; the calls that do GPU work
(objective and trial-step values, gradients, K-metric dot products) post a
work item to the engine and wait for its result.  The engine loop:

  1. admits arrived requests while the HBM budget and the slot count allow;
     an admitted request's momenta, trajectories and optimiser directions
     stay on the device until it finishes;
  2. waits until every active request has posted its next work item;
  3. runs each kind of pending work as ONE ragged launch over all requests
     that posted it (lddmm_ragged_* entry points: segment tables with
     per-request offsets, kernel widths and source-chunk counts);
  4. hands the results back and repeats.

Requests that arrive while others are on the GPU are admitted at once and join
the next launches, so their work overlaps on the device.  Every per-request
quantity (packing frame, source chunking, reduction trees, line-search
decisions) depends only on that request's own data, so a request's result is
bit-identical alone and in any mix.

Precision: FP32 compensated kernel sums for shooting, the adjoint, the data
term and the dot products; every energy and dot product is reduced in FP64.
The line search of the reference compares objective values down to an
absolute 1e-6 (its stop test and its tiny `epsSmall` probe step), while the
objective is a small difference of norms of order |S|^2 / sigmaError^2.
``line_search_precision``:
  'auto' (default): trial values use FP32c data-term sums and carry an error
      bound; a comparison that the bounds cannot decide re-evaluates the data
      term of both values in FP64 (registration_b200._precision), so every
      decision is the one an FP64 evaluation takes;
  'fp64': every trial value uses an FP64 data-term sweep;
  'fp32c': no refinement (fastest; decisions between values closer than the
      FP32c noise are arbitrary, which can end a run early).
"""
import threading
import time

import numpy as np
import torch

from . import _dataterm as _dt
from . import _lib
from . import _ragged as _rg
from . import conjugateGradient as cg
from ._precision import _Value, value_bound
from .device import require_cuda

NORMS = _rg.NORMS


class RequestCancelled(Exception):
    """A request withdrawn with MatchRequest.cancel()."""


class ServingStopped(RuntimeError):
    """The engine stopped (its run() left on an exception) before the request ended."""


def _volume(v, f):
    """Signed volume sum_f det(v0, v1, v2) / 6 (surfaces.py:711-717)."""
    return float((np.linalg.det(v[f]) / 6).sum())


class MatchRequest:
    """One matching problem.

    Template / Target: surfaces.Surface or curves.Curve (vertices, faces);
    param: SurfaceMatchingParam / CurveMatchingParam (timeStep, KparDiff,
    KparDist, sigmaError, errorType); maxIter / regWeight as in
    SurfaceMatching; verb is the matching classes' verb, passed to cg (it
    selects cg's branch after a failed tiny step, conjugateGradient.py:151-154);
    at_init: initial momenta (T, n, d), zero when None (SurfaceMatching starts
    from zero, surfaceMatching.py:110).  cancel() withdraws the request: a
    queued request is dropped, an active one stops at its next GPU call; both
    end with a RequestCancelled error and free their slot and budget.
    The kernels' sigma / name / order are used; the kernel sums run in FP32
    with compensated accumulation whatever their precision."""

    def __init__(self, Template, Target, param, maxIter=50, regWeight=1.0, rid=None, verb=True, at_init=None):
        if param.errorType not in NORMS:
            raise ValueError("errorType must be one of %s" % sorted(NORMS))
        self.v0 = np.ascontiguousarray(np.asarray(Template.vertices, dtype=np.float64))
        self.f0 = np.ascontiguousarray(np.asarray(Template.faces, dtype=np.int64))
        self.v1 = np.ascontiguousarray(np.asarray(Target.vertices, dtype=np.float64))
        self.f1 = np.ascontiguousarray(np.asarray(Target.faces, dtype=np.int64))
        if self.f0.shape[1] != self.f1.shape[1] or self.v0.shape[1] != self.v1.shape[1]:
            raise ValueError("template and target must have the same cell size and dimension")
        if param.errorType == "varifold" and self.f0.shape[1] != 3:
            raise ValueError("the varifold norm is defined for triangulated surfaces")
        if self.f0.shape[1] == 3 and self.v0.shape[1] == 3 and np.isfinite(self.v0).all() \
                and np.isfinite(self.v1).all():
            # SurfaceMatching orients the target like the template (surfaceMatching.py:126-129)
            if _volume(self.v0, self.f0) * _volume(self.v1, self.f1) < 0:
                self.f1 = np.ascontiguousarray(self.f1[:, [0, 2, 1]])
        # cg's first step: SurfaceMatching passes epsInit = 0.1 (surfaceMatching.py:484),
        # CurveMatching keeps cg's default 10 (curveMatching.py:352)
        self.eps_init = 0.1 if self.f0.shape[1] == 3 else 10.0
        self.param = param
        self.T = int(round(1.0 / param.timeStep))
        self.max_iter = int(maxIter)
        self.regweight = float(regWeight)
        self.verb = bool(verb)
        self.at_init = None
        if at_init is not None:
            self.at_init = np.ascontiguousarray(np.asarray(at_init, dtype=np.float64))
            if self.at_init.shape != (self.T, len(self.v0), self.v0.shape[1]):
                raise ValueError("at_init must be (T, n, d) = %s" % ((self.T, len(self.v0), self.v0.shape[1]),))
        self.cancelled = False
        self.rid = rid
        self.arrival = None
        self.start = None
        self.finish = None
        self.result = None
        self.error = None
        self.done = threading.Event()

    @property
    def n(self):
        return len(self.v0)

    def cancel(self):
        """Withdraws the request (see the class docstring)."""
        self.cancelled = True

    def input_error(self):
        """ValueError for inputs no solve can start from (non-finite vertices or
        initial momenta, cell indices out of range), else None."""
        for name, a in (("template vertices", self.v0), ("target vertices", self.v1),
                        ("initial momenta", self.at_init)):
            if a is not None and not np.isfinite(a).all():
                return ValueError("request %s: %s are not finite" % (self.rid, name))
        for name, f, v in (("template", self.f0, self.v0), ("target", self.f1, self.v1)):
            if f.size and (f.min() < 0 or f.max() >= len(v)):
                return ValueError("request %s: %s cell indices out of range" % (self.rid, name))
        return None

    @property
    def group(self):
        """Requests of one group can share a ragged launch."""
        p = self.param
        return (self.v0.shape[1], self.f0.shape[1], p.errorType, _rg.kernel_order(p.KparDiff), _rg.kernel_order(p.KparDist), self.T)

    def hbm_bytes(self):
        """Resident device state: momenta, trial momenta, gradient and three
        optimiser directions (T n d each), two trajectories and the adjoint
        ((T+1) n d each), target cells and topology, plus a share of the
        ragged launches' packed records."""
        n, d, T = self.n, self.v0.shape[1], self.T
        cells = len(self.f0) + len(self.f1)
        return 8 * (7 * T * n * d + 4 * (T + 1) * n * d) + 160 * cells + 96 * n * (T + 2)

    def latency(self):
        return None if self.finish is None else self.finish - self.arrival


class _Direction:
    __slots__ = ("diff", "aff", "initx")

    def __init__(self, diff):
        self.diff = diff
        self.aff = np.zeros((0,))
        self.initx = []


class _Problem:
    """The optimiser protocol (surfaceMatching.py:233-377) of one request; the
    GPU work is posted to the engine."""

    def __init__(self, req, engine):
        self.req = req
        self.engine = engine
        dev = engine.device
        p = req.param
        self.T = self.Tsize = req.T
        self.dim = req.v0.shape[1]
        self.npt = req.n
        self.sigma_def = float(p.KparDiff.sigma)
        self.sigma_dist = float(p.KparDist.sigma)
        self.s2 = float(p.sigmaError) ** 2
        self.x0 = torch.from_numpy(req.v0).to(dev)
        self.v1 = torch.from_numpy(req.v1).to(dev)
        c1, s1 = _dt.cell_geometry(req.v1, req.f1)
        self.tc = torch.from_numpy(np.ascontiguousarray(c1)).to(dev)
        self.tv = torch.from_numpy(np.ascontiguousarray(s1)).to(dev)
        # fixed data-term packing frame: centre of the target cells' bounding box
        lo, hi = c1.min(axis=0), c1.max(axis=0)
        self.frame = tuple(float(0.5 * (lo[j] + hi[j])) if j < c1.shape[1] else 0.0 for j in range(3))
        self.noise_obs = 0.0
        self.dshape = _dt.DeviceShape(req.f0, req.n)
        self.tshape = _dt.DeviceShape(req.f1, len(req.v1))
        if req.at_init is None:
            self.at = torch.zeros((self.T, self.npt, self.dim), dtype=torch.float64, device=dev)
        else:
            self.at = torch.from_numpy(req.at_init).to(dev)
        self.atTry = self.at
        self.xt = self.x0.unsqueeze(0).repeat(self.T + 1, 1, 1)
        self.xtTry = None
        self.obj = None
        self.objTry = None
        self.obj0 = None
        self.gradCoeff = self.npt
        self.converged = False
        self.iters = 0
        self.calls = {"value": 0, "grad": 0, "dot": 0, "refine": 0}

    def getVariable(self):
        return [self.at]

    def _value(self, at):
        """obj0 + deformation energy + data term / sigmaError^2 at momenta `at`."""
        tot, ereg, xt = self.engine.post(self, "value", at)
        v = self.obj0 + tot
        if self.engine.lsp == "auto":
            v = _Value(v, self, ereg, xt[-1], value_bound(self, self.engine.noise, self.obj0))
        return v, xt

    def exact_value(self, ereg, x_end):
        """The same objective with an FP64 data-term value (one posted launch)."""
        return self.obj0 + ereg + self.engine.post(self, "refine", x_end)

    def objectiveFun(self):
        if self.obj is None:
            self.obj0 = self.engine.post(self, "norm0", None)
            self.obj, self.xt = self._value(self.at)
            # the reference maps a NaN trial to 1e500 (surfaceMatching.py:278-280), which
            # rejects that step; a non-finite starting objective has no step to reject
            if not np.isfinite(float(self.obj)):
                raise FloatingPointError("request %s: the objective at the initial momenta is not finite"
                                         % self.req.rid)
        return self.obj

    def updateTry(self, dir, eps, objRef=None):
        atTry = self.at - eps * dir.diff
        objTry, xt = self._value(atTry)
        if np.isnan(objTry):
            return 1e500
        if (objRef is None) or (objTry < objRef):
            self.atTry = atTry
            self.objTry = objTry
            self.xtTry = xt
        return objTry

    def getGradient(self, coeff=1.0):
        dat = self.engine.post(self, "grad", None)
        return _Direction(dat / (coeff * self.T))

    def dotProduct(self, g1, g2):
        return self.engine.post(self, "dot", (g1.diff, [g.diff for g in g2]))

    def addProd(self, d1, d2, beta):
        return _Direction(d1.diff + beta * d2.diff)

    def copyDir(self, d0):
        return _Direction(d0.diff.clone())

    def acceptVarTry(self):
        self.obj = self.objTry
        self.at = self.atTry
        if self.xtTry is not None:
            self.xt = self.xtTry

    def endOfIteration(self):
        self.iters += 1


class _Lane:
    """One size class of requests: its own round loop (thread) and, on the GPU,
    its own CUDA stream (smaller requests: higher stream priority)."""

    def __init__(self, idx, bound):
        self.idx = idx
        self.bound = bound
        self.active = set()
        self.pending = {}        # problem -> (kind, payload)
        self.rounds = 0
        self.stream = None
        self.thread = None


class Scheduler:
    """Admission, lanes, rounds and grouping of the continuous-batching loop.

    Subclasses provide _make_problem(req) and one _do_<kind>(items) method per
    kind of work ("norm0", "value", "grad", "dot"), each mapping a list of
    (problem, payload) to a list of results (one launch per call), and may
    override _lane_context(lane) (the context a lane's work runs in).

    hbm_budget_bytes: admission limit on the sum of the active requests'
    resident state (MatchRequest.hbm_bytes); max_active: slot count;
    lanes: increasing request-size bounds (vertex counts) of the size classes,
    the last one unbounded, e.g. (5000, 16000) -> three lanes.  Each lane waits
    for its own requests only, so small requests are not held back by the
    rounds of large ones."""

    def __init__(self, hbm_budget_bytes=150e9, max_active=64, lanes=()):
        self.hbm_budget = float(hbm_budget_bytes)
        self.max_active = int(max_active)
        bounds = sorted(float(b) for b in lanes) + [float("inf")]
        self.lanes = [_Lane(k, b) for k, b in enumerate(bounds)]
        self.cv = threading.Condition()
        self.stats_lock = threading.Lock()
        self.queue = []          # submitted, not admitted (sorted by arrival)
        self.results = {}
        self.events = {}
        self.finished = []
        self.hbm_in_use = 0.0
        self.n_active = 0
        self.rounds = 0
        self.launches = {"norm0": 0, "value": 0, "grad": 0, "dot": 0, "refine": 0}
        self.batch_sizes = []
        self.busy_seconds = 0.0
        self.max_active_seen = 0
        self.peak_hbm = 0.0
        self.threads = []
        self._stop = False

    def _lane_of(self, req):
        return next(l for l in self.lanes if req.n <= l.bound)

    def _lane_context(self, lane):
        import contextlib
        return contextlib.nullcontext()

    # -- request side ------------------------------------------------------------------
    def submit(self, req, arrival=None):
        """Queues a request; `arrival` (perf_counter seconds) may lie in the future."""
        req.arrival = time.perf_counter() if arrival is None else float(arrival)
        with self.cv:
            self.queue.append(req)
            self.queue.sort(key=lambda r: r.arrival)
            self.cv.notify_all()
        return req

    def post(self, prob, kind, payload):
        if getattr(prob.req, "cancelled", False):
            raise RequestCancelled("request %s cancelled" % prob.req.rid)
        ev = threading.Event()
        with self.cv:
            if self._stop:
                raise ServingStopped("the engine has stopped")
            self.events[prob] = ev
            prob.lane.pending[prob] = (kind, payload)
            self.cv.notify_all()
        ev.wait()
        res = self.results.pop(prob)
        if isinstance(res, BaseException):
            raise res
        if getattr(prob.req, "cancelled", False):
            raise RequestCancelled("request %s cancelled" % prob.req.rid)
        return res

    def _run_request(self, req, lane, slot):
        """Request thread: builds the problem in its lane's context and runs the
        optimiser.  `slot` is the placeholder counted active until the problem
        exists."""
        prob = None
        try:
            with self._lane_context(lane):
                prob = self._make_problem(req)
                prob.lane = lane
                with self.cv:
                    lane.active.discard(slot)
                    lane.active.add(prob)
                    self.cv.notify_all()
                # SurfaceMatching / CurveMatching.optimizeMatching (surfaceMatching.py:474-484,
                # curveMatching.py:342-352: gradEps = max(1e-3, |g| / 1e4))
                grd = prob.getGradient(prob.gradCoeff)
                [g2] = prob.dotProduct(grd, [grd])
                prob.gradEps = max(0.001, np.sqrt(g2) / 10000)
                cg.cg(prob, verb=getattr(req, "verb", True), maxIter=req.max_iter, TestGradient=False,
                      epsInit=getattr(req, "eps_init", 0.1))
                obj = prob.obj.refine() if isinstance(prob.obj, _Value) else float(prob.obj)
                req.result = {"at": prob.at, "xt": prob.xt, "obj": obj, "iters": prob.iters,
                              "converged": prob.converged, "calls": dict(prob.calls)}
                self._request_done(prob)
        except BaseException as exc:   # this request fails, the others go on
            req.error = exc
        finally:
            req.finish = time.perf_counter()
            with self.cv:
                lane.active.discard(slot)
                lane.active.discard(prob)
                self.n_active -= 1
                self.hbm_in_use -= req.hbm_bytes()
                self.finished.append(req)
                self.cv.notify_all()
            req.done.set()

    def _request_done(self, prob):
        """Hook: the request's last results are final (e.g. wait for its stream)."""

    # -- admission (main thread) --------------------------------------------------------
    def _admit(self, now):
        start = []
        with self.cv:
            keep = []
            for req in self.queue:
                bad = RequestCancelled("request %s cancelled" % req.rid) if getattr(req, "cancelled", False) else None
                if bad is None and req.arrival <= now and hasattr(req, "input_error"):
                    bad = req.input_error()
                if bad is not None:
                    req.error = bad
                    req.start = req.finish = now
                    self.finished.append(req)
                    req.done.set()
                elif req.arrival > now:
                    keep.append(req)
                elif req.hbm_bytes() > self.hbm_budget:
                    req.error = MemoryError("request needs %.3g bytes of device state; the budget is %.3g"
                                            % (req.hbm_bytes(), self.hbm_budget))
                    req.start = req.finish = now
                    self.finished.append(req)
                    req.done.set()
                elif (self.n_active + len(start) < self.max_active
                      and self.hbm_in_use + req.hbm_bytes() <= self.hbm_budget):
                    self.hbm_in_use += req.hbm_bytes()
                    self.peak_hbm = max(self.peak_hbm, self.hbm_in_use)
                    start.append(req)
                else:
                    keep.append(req)
            self.queue = keep
            for req in start:
                lane = self._lane_of(req)
                slot = object()
                lane.active.add(slot)
                self.n_active += 1
                self.max_active_seen = max(self.max_active_seen, self.n_active)
                req.start = time.perf_counter()
                th = threading.Thread(target=self._run_request, args=(req, lane, slot), daemon=True)
                self.threads.append(th)
                th.start()
        return len(start)

    def _can_admit(self, now):
        if not self.queue or self.queue[0].arrival > now:
            return False
        req = self.queue[0]
        return (self.n_active < self.max_active
                and (self.hbm_in_use + req.hbm_bytes() <= self.hbm_budget or req.hbm_bytes() > self.hbm_budget))

    # -- lanes ------------------------------------------------------------------------------
    def _lane_loop(self, lane):
        with self._lane_context(lane):
            while True:
                with self.cv:
                    while not (lane.active and len(lane.pending) == len(lane.active)) and not self._stop:
                        self.cv.wait()
                    if not (lane.active and len(lane.pending) == len(lane.active)):
                        return
                    ready = lane.pending
                    lane.pending = {}
                t0 = time.perf_counter()
                try:
                    self._execute(ready)
                except BaseException as exc:   # e.g. KeyboardInterrupt in a launch
                    self._fail_waiting(ready, exc)
                    raise
                with self.stats_lock:
                    self.busy_seconds += time.perf_counter() - t0
                    self.rounds += 1
                    lane.rounds += 1

    def run(self):
        """Serves until the queue (including future arrivals) and every lane are empty."""
        self._stop = False
        for lane in self.lanes:
            lane.thread = threading.Thread(target=self._lane_loop, args=(lane,), daemon=True)
            lane.thread.start()
        try:
            while True:
                self._admit(time.perf_counter())
                with self.cv:
                    if self.n_active == 0 and not self.queue:
                        break
                    now = time.perf_counter()
                    if self._can_admit(now):
                        continue
                    nxt = self.queue[0].arrival if self.queue else None
                    wait = None if (nxt is None or nxt <= now) else nxt - now
                    self.cv.wait(timeout=wait)
        finally:
            with self.cv:
                self._stop = True
                self.cv.notify_all()
            for lane in self.lanes:
                lane.thread.join()
            # on a normal exit every request has ended; after an exception, fail the
            # requests still queued or waiting for a round so their threads end
            with self.cv:
                stopped = ServingStopped("the engine stopped before the request ended")
                for req in self.queue:
                    req.error = stopped
                    req.finish = time.perf_counter()
                    self.finished.append(req)
                    req.done.set()
                self.queue = []
                waiting = {}
                for lane in self.lanes:
                    waiting.update(lane.pending)
                    lane.pending = {}
            self._fail_waiting(waiting, stopped)
            for th in self.threads:
                th.join()
            self.threads = []

    def _fail_waiting(self, items, exc):
        """Hands `exc` to the request threads blocked in post() for `items`."""
        with self.cv:
            for prob in list(items):
                ev = self.events.pop(prob, None)
                if ev is not None:
                    self.results[prob] = exc
                    ev.set()

    def _execute(self, ready):
        groups = {}
        for prob, (kind, payload) in ready.items():
            groups.setdefault((kind, prob.req.group), []).append((prob, payload))
        with self.stats_lock:
            self.batch_sizes.append(len(ready))
        out = {}
        for (kind, _), items in groups.items():
            with self.stats_lock:
                self.launches[kind] += 1
            fn = getattr(self, "_do_" + kind)
            try:
                res = fn(items)
            except Exception as exc:
                # isolate the failing request(s): re-run the group one by one
                res = [exc] * len(items)
                if len(items) > 1:
                    for j, it in enumerate(items):
                        try:
                            res[j] = fn([it])[0]
                        except Exception as exc1:
                            res[j] = exc1
            for (prob, _), r in zip(items, res):
                out[prob] = r
        for prob, r in out.items():
            self.results[prob] = r
            self.events.pop(prob).set()

    # -- reporting -------------------------------------------------------------------------
    def stats(self):
        lat = np.array([r.latency() for r in self.finished if r.error is None])
        return {"finished": len(self.finished), "failed": sum(r.error is not None for r in self.finished),
                "rounds": self.rounds, "lane_rounds": [l.rounds for l in self.lanes],
                "launch_groups": dict(self.launches),
                "mean_batch": float(np.mean(self.batch_sizes)) if self.batch_sizes else 0.0,
                "max_batch": int(max(self.batch_sizes)) if self.batch_sizes else 0,
                "max_active": self.max_active_seen, "peak_hbm_bytes": self.peak_hbm,
                "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
                "p99_s": float(np.percentile(lat, 99)) if lat.size else None}


class ServingEngine(Scheduler):
    """Continuous-batching matcher on the current CUDA device: submit() from any
    thread, run() drives the GPU.

    Each lane (size class, see Scheduler) launches on its own CUDA stream; the
    lane of the smallest requests has the highest stream priority, so the
    block scheduler runs its short kernels between the blocks of the large
    requests' sweeps.  line_search_precision: 'auto' (default), 'fp64' or
    'fp32c', see the module docstring; noise: the initial bound of the error
    of a difference of two FP32c objective values, as a fraction of the
    target's Norm0 / sigmaError^2 (measured near optima: ~1e-9 of it; the
    bound grows with every error measured by a refinement); fixed_frame: pack
    each request's data term relative to a fixed centre (the target's
    bounding box), so values of different calls share the rounding of the
    target cells."""

    def __init__(self, hbm_budget_bytes=150e9, max_active=64, line_search_precision="auto",
                 lanes=(5000, 16000), fixed_frame=True, noise=1e-8):
        require_cuda()
        _lib.load()
        if line_search_precision not in ("auto", "fp32c", "fp64"):
            raise ValueError("line_search_precision must be 'auto', 'fp32c' or 'fp64'")
        super().__init__(hbm_budget_bytes, max_active, lanes)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.lsp = line_search_precision
        self.fixed_frame = bool(fixed_frame)
        self.noise = float(noise)
        least, greatest = torch.cuda.Stream.priority_range()
        nl = len(self.lanes)
        for lane in self.lanes:
            prio = max(greatest, least - (nl - 1 - lane.idx))
            lane.stream = torch.cuda.Stream(device=self.device, priority=prio)

    def _lane_context(self, lane):
        return torch.cuda.stream(lane.stream)

    def _make_problem(self, req):
        return _Problem(req, self)

    def run(self):
        # the lanes' streams start after everything queued on the caller's stream
        for lane in self.lanes:
            lane.stream.wait_stream(torch.cuda.current_stream())
        super().run()
        for lane in self.lanes:
            torch.cuda.current_stream().wait_stream(lane.stream)

    # -- ragged operations -----------------------------------------------------------------
    def _dataterm(self, probs, verts, grad, precision, target_self=False, frame=True):
        """Ragged data term (lddmm_ragged_dataterm_*): NormDef values, Norm0 of
        the targets (target_self) or NormGradient w.r.t. the vertices."""
        req0 = probs[0].req
        return _rg.dataterm(req0.param.errorType, verts, [p.tshape if target_self else p.dshape for p in probs],
                            None if target_self else [p.tc for p in probs],
                            None if target_self else [p.tv for p in probs],
                            [p.sigma_dist for p in probs], _rg.kernel_order(req0.param.KparDist), precision, grad,
                            frames=[p.frame for p in probs] if (frame and self.fixed_frame) else None)

    def _value_precision(self):
        return "fp64" if self.lsp == "fp64" else "fp32c"

    def _do_norm0(self, items):
        """Norm0 of the targets (a constant of each request): FP64 unless the
        line search is all-FP32c."""
        probs = [p for p, _ in items]
        prec = "fp32c" if self.lsp == "fp32c" else "fp64"
        e = self._dataterm(probs, [p.v1 for p in probs], False, prec, target_self=True).cpu().numpy()
        return [float(e[i]) / p.s2 for i, p in enumerate(probs)]

    def _do_refine(self, items):
        """FP64 data term / sigmaError^2 at stored end points (the 'auto' line search)."""
        probs = [p for p, _ in items]
        D = self._dataterm(probs, [x for _, x in items], False, "fp64")
        s2 = torch.tensor([p.s2 for p in probs], dtype=torch.float64, device=self.device)
        out = (D / s2).cpu().numpy()
        for p in probs:
            p.calls["refine"] += 1
        return [float(out[i]) for i in range(len(probs))]

    def _do_value(self, items):
        """Shooting + deformation energy (lddmm_ragged_shoot_f32c), then the data
        term at the end points: objectiveFunDef + dataTerm (surfaceMatching.py:187-231)."""
        probs = [p for p, _ in items]
        T, d = probs[0].T, probs[0].dim
        v_off = _rg.offsets([p.npt for p in probs])
        XT, E = _rg.shoot(torch.cat([p.x0 for p in probs]), torch.cat([a.reshape(-1, d) for _, a in items]),
                          v_off, T, [p.sigma_def for p in probs], _rg.kernel_order(probs[0].req.param.KparDiff),
                          [p.req.regweight for p in probs])
        xts = [XT[(T + 1) * v_off[i]:(T + 1) * v_off[i + 1]].view(T + 1, p.npt, d) for i, p in enumerate(probs)]
        D = self._dataterm(probs, [xt[-1] for xt in xts], False, self._value_precision())
        s2 = torch.tensor([p.s2 for p in probs], dtype=torch.float64, device=self.device)
        host = torch.stack([E + D / s2, E]).cpu().numpy()
        for p in probs:
            p.calls["value"] += 1
        return [(float(host[0, i]), float(host[1, i]), xts[i]) for i in range(len(probs))]

    def _do_grad(self, items):
        """grd.diff = (2 rw a - p_{t+1}) from the adjoint with p_T = -grad D / sigmaError^2
        (surfaceMatching.py:301-327, pointEvolution.py:735-817)."""
        probs = [p for p, _ in items]
        T, d = probs[0].T, probs[0].dim
        pxs = self._dataterm(probs, [p.xt[-1] for p in probs], True, "fp32c")
        v_off = _rg.offsets([p.npt for p in probs])
        _, DAT = _rg.covector(torch.cat([p.xt.reshape(-1, d) for p in probs]),
                              torch.cat([p.at.reshape(-1, d) for p in probs]),
                              torch.cat([px / (-p.s2) for p, px in zip(probs, pxs)]), v_off, T,
                              [p.sigma_def for p in probs], _rg.kernel_order(probs[0].req.param.KparDiff),
                              [p.req.regweight for p in probs])
        for p in probs:
            p.calls["grad"] += 1
        return [DAT[T * v_off[i]:T * v_off[i + 1]].view(T, p.npt, d) for i, p in enumerate(probs)]

    def _do_dot(self, items):
        """sum_t <g2_t, K(x_t) g1_t> for every g2 (surfaceMatching.py:353-377):
        one applyK segment per (request, t) in a single ragged launch."""
        probs = [p for p, _ in items]
        T, d = probs[0].T, probs[0].dim
        XT = torch.cat([p.xt[:T].reshape(-1, d) for p in probs])
        G1 = torch.cat([g1.reshape(-1, d) for _, (g1, _) in items])
        starts, counts, sig = [], [], []
        row = 0
        for p in probs:
            for t in range(T):
                starts.append(row + t * p.npt)
                counts.append(p.npt)
                sig.append(p.sigma_def)
            row += T * p.npt
        U = _rg.applyk_segments(XT, G1, starts, counts, sig, _rg.kernel_order(probs[0].req.param.KparDiff))
        outs = []
        row = 0
        for p, (_, g2s) in items:
            u = U[row:row + T * p.npt].reshape(-1)
            row += T * p.npt
            G2 = torch.stack([g.reshape(-1) for g in g2s])
            outs.append(G2 @ u)
            p.calls["dot"] += 1
        host = torch.cat(outs).cpu().numpy()
        res, k = [], 0
        for _, (_, g2s) in items:
            res.append(host[k:k + len(g2s)].copy())
            k += len(g2s)
        return res


def serve(requests, **engine_kw):
    """Runs a list of requests (arrival times already set, or now) to completion."""
    eng = ServingEngine(**engine_kw)
    for r in requests:
        eng.submit(r, arrival=r.arrival)
    eng.run()
    return eng
