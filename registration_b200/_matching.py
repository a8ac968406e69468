"""Device-resident implementation of the matching-problem protocol shared by
SurfaceMatching (py-lddmm/surfaceMatching.py:74-486) and CurveMatching
(py-lddmm/curveMatching.py:58-354): objectiveFunDef / objectiveFun /
updateTry / getGradient / dotProduct / acceptVarTry / endOfIteration.

Momenta, trajectory, directions and shapes stay on the GPU (FP64 storage);
every objective value and dot product is reduced in FP64 on the device and
read back as one host double, which is what the line search compares.

Precision: kernel sums (shooting, adjoint, data-term gradient, dot products)
follow the kernels' own precision.  The reference's stop test is an absolute
|obj - objTry| < 1e-6 on objectives that are differences of norms of order
|S|^2 (1e2 for a unit sphere at sigmaError 0.5), i.e. ~1e-9 relative, which
FP32 pair evaluation cannot always resolve.  lineSearchPrecision selects the
data-term VALUE that the line search compares:
  'fp64' (default): an FP64 copy of KparDist for every value;
  'auto': KparDist's own precision with an error bound, refined to FP64 only
      when a comparison cannot be decided (registration_b200._precision);
  'fp32c' / KparDist's precision: no refinement.

Two reuses that do not change any value: the trajectory of an accepted trial
step is kept instead of re-shooting it in endOfIteration, and getGradient
runs the adjoint on that stored trajectory instead of re-shooting inside
landmarkHamiltonianGradient (the shots are deterministic, so they would be
bit-identical).

With cudaGraphs (the default) the trial steps are replayed from a CUDA graph;
for problems small enough to run on one thread-block cluster a replay
evaluates a batch of the step sizes the line search asks for next (one
cluster each, side by side), and the gradient is replayed from a second
graph.  Every value, and so every decision and the accepted trace, equals
the eager path's.
"""
import contextlib
import gc
import logging

import numpy as np
import torch

from . import _dataterm as _dt
from . import _ragged as _rg
from . import pointEvolution as evol
from ._precision import _Value, value_bound
from .device import require_cuda, to_dev, workspace


@contextlib.contextmanager
def _gc_paused():
    """Python's cycle collector paused while a CUDA graph is captured: a
    collection that falls inside the capture costs milliseconds and frees
    nothing the capture needs."""
    was = gc.isenabled()
    gc.disable()
    try:
        yield
    finally:
        if was:
            gc.enable()


class Direction:
    def __init__(self):
        self.diff = []
        self.aff = []
        self.initx = []


class DeviceMatching:
    """Subclasses set: fv0, fv1 (shapes), param, norm_name, tgt_vectors_attr."""

    # The best trial step's momenta and trajectory.  A batched trial leaves them
    # in a slot of the batch buffers; they are copied out only when read, when
    # accepted, or before the next batch overwrites the slot.
    _pending_try = None

    def _materialize_try(self):
        pend = self._pending_try
        if pend is not None:
            g, b = pend
            self._pending_try = None
            self.__dict__["_atTry"] = g["atTry"][b].clone()
            self.__dict__["_xtTry"] = g["xt"][b].clone()

    @property
    def atTry(self):
        self._materialize_try()
        return self.__dict__.get("_atTry")

    @atTry.setter
    def atTry(self, v):
        self._materialize_try()
        self.__dict__["_atTry"] = v

    @property
    def xtTry(self):
        self._materialize_try()
        return self.__dict__.get("_xtTry")

    @xtTry.setter
    def xtTry(self, v):
        self._materialize_try()
        self.__dict__["_xtTry"] = v

    def _init_state(self, maxIter, regWeight, verb, testGradient, affine, symmetric, lineSearchPrecision='fp64',
                    noise=1e-8, cudaGraphs=True):
        require_cuda()
        if affine not in ('none', None):
            raise NotImplementedError("affine registration components are not provided (affine='none' only)")
        if symmetric:
            raise NotImplementedError("symmetric matching is not provided")
        self.maxIter = maxIter
        self.verb = verb
        self.testGradient = testGradient
        self.regweight = regWeight
        self.affine = 'none'
        self.affineDim = 0
        self.symmetric = False
        self.iter = 0
        self.Tsize = int(round(1.0 / self.param.timeStep))
        self.x0 = to_dev(self.fv0.vertices)
        self.npt, self.dim = self.x0.shape
        dev = self.x0.device
        self.at = torch.zeros((self.Tsize, self.npt, self.dim), dtype=torch.float64, device=dev)
        self.atTry = self.at.clone()
        self.Afft = np.zeros((self.Tsize, 0))
        self.AfftTry = self.Afft
        self.xt = self.x0.unsqueeze(0).repeat(self.Tsize + 1, 1, 1)
        self.xtTry = None
        self.calls = {"updateTry": 0, "getGradient": 0, "dotProduct": 0}
        self.cudaGraphs = bool(cudaGraphs)
        self._graph = None
        self._grad_graph = None
        self.obj = None
        self.objTry = None
        self.gradCoeff = self.npt
        self._dshape = self.fv0.device_shape()
        self._tc = to_dev(self.fv1.centers)
        self._tv = to_dev(getattr(self.fv1, self.tgt_vectors_attr))
        self.fvDef.updateVertices(self.x0)
        self._fast_data = self._our_norm_functions()
        K = self.param.KparDist
        self._auto = lineSearchPrecision == 'auto'
        self._noise = float(noise)
        self.noise_obs = 0.0
        self._K64 = K if K.precision == 'fp64' else type(K)(name=K.name, sigma=K.sigma, order=K.order,
                                                              weight=K.weight, precision='fp64')
        if self._auto or lineSearchPrecision == K.precision:
            self._Kval = K
        else:
            self._Kval = type(K)(name=K.name, sigma=K.sigma, order=K.order, weight=K.weight,
                                 precision=lineSearchPrecision)

    # -- data term ------------------------------------------------------------
    def _our_norm_functions(self):
        """True when param's (fun_obj0, fun_obj, fun_objGrad) are this library's
        own norms, so the device path can be used directly."""
        mod = self.norm_module
        name = getattr(self.param, 'errorType', None)
        if name not in ('current', 'measure', 'varifold'):
            return False
        want = (getattr(mod, name + 'Norm0', None), getattr(mod, name + 'NormDef', None),
                getattr(mod, name + 'NormGradient', None))
        return (self.param.fun_obj0, self.param.fun_obj, self.param.fun_objGrad) == want

    def _data_raw(self, vertices, K=None, out=None):
        """fun_obj(fvDef, fv1, KparDist) (not yet divided by sigmaError^2) as a
        device scalar; the fast path writes it into the 0-d tensor `out` if given."""
        K = self._Kval if K is None else K
        if self._fast_data:
            e, _ = _dt.dataterm(self.param.errorType, vertices, self._dshape, self._tc, self._tv,
                                K, energy=True, grad=False, energy_out=out)
            return e
        ff = self.shape_copy(self.fvDef)
        ff.updateVertices(vertices)
        e = torch.tensor(self.param.fun_obj(ff, self.fv1, K), dtype=torch.float64, device=self.x0.device)
        if out is not None:
            out.copy_(e)
            return out
        return e

    def _data_energy(self, vertices, K=None):
        """fun_obj(fvDef, fv1, KparDist) / sigmaError^2 as a device scalar."""
        return self._data_raw(vertices, K) / (self.param.sigmaError ** 2)

    def _combine(self, ereg, data_raw):
        """obj0 + deformation energy + data term / sigmaError^2 from host doubles
        (one formula for the eager, graphed and refined values)."""
        return self.obj0 + (ereg + data_raw / self.param.sigmaError ** 2)

    def _trial_value(self, e_reg, x_end):
        """obj0 + deformation energy + data term, as compared by the line search."""
        host = torch.stack([e_reg, self._data_raw(x_end)]).cpu().numpy()
        ereg = float(host[0])
        v = self._combine(ereg, float(host[1]))
        if self._auto:
            v = _Value(v, self, ereg, x_end, value_bound(self, self._noise, self.obj0))
        return v

    def exact_value(self, ereg, x_end):
        """The objective with an FP64 data-term value (refinement of a _Value)."""
        self.calls["refine"] = self.calls.get("refine", 0) + 1
        return self._combine(ereg, float(self._data_raw(x_end, self._K64)))

    def dataTerm(self, _fvDef, _fvInit=None):
        return float(self._data_energy(to_dev(_fvDef.vertices)))

    def endPointGradient(self):
        return self._end_point_gradient(self.xt[-1])

    def _end_point_gradient(self, x_end):
        if self._fast_data:
            _, px = _dt.dataterm(self.param.errorType, x_end, self._dshape, self._tc, self._tv,
                                 self.param.KparDist, energy=False, grad=True)
        else:
            px = to_dev(self.param.fun_objGrad(self.fvDef, self.fv1, self.param.KparDist))
        return px / self.param.sigmaError ** 2

    # -- objective --------------------------------------------------------------
    def objectiveFunDef(self, at, Afft=None, withTrajectory=False, withJacobian=False, x0=None):
        """Deformation cost sum_t rw dt <a_t, K(x_t) a_t> (surfaceMatching.py:187-221)."""
        x0 = self.x0 if x0 is None else to_dev(x0)
        xt, e = evol.shoot(x0, to_dev(at), self.param.KparDiff, regweight=self.regweight, with_energy=True)
        obj = float(e)
        if withJacobian:
            _, Jt = evol.landmarkDirectEvolutionEuler(x0, to_dev(at), self.param.KparDiff, withJacobian=True)
            return obj, xt, Jt
        if withTrajectory:
            return obj, xt
        return obj

    def objectiveFun(self):
        """(surfaceMatching.py:233-250)"""
        if self.obj is None:
            K0 = self._K64 if self._auto else self._Kval
            self.obj0 = self.param.fun_obj0(self.fv1, K0) / (self.param.sigmaError ** 2)
            xt, e = evol.shoot(self.x0, self.at, self.param.KparDiff, regweight=self.regweight, with_energy=True)
            self.xt = xt
            self.fvDef.updateVertices(xt[-1])
            self.obj = self._trial_value(e, xt[-1])
        return self.obj

    def getVariable(self):
        return [self.at, self.Afft]

    def updateTry(self, dir, eps, objRef=None):
        """(surfaceMatching.py:255-289); NaN objectives return 1e500."""
        self.calls["updateTry"] += 1
        if self.cudaGraphs and self._fast_data:
            return self._graph_update_try(dir, eps, objRef)
        eps_d = torch.full((), float(eps), dtype=torch.float64, device=self.x0.device)
        atTry, xt, e = evol.shoot_along(self.x0, self.at, dir.diff, eps_d, self.param.KparDiff,
                                        regweight=self.regweight)
        objTry = self._trial_value(e, xt[-1])
        if np.isnan(objTry):
            logging.info('Warning: nan in updateTry')
            return 1e500
        if (objRef is None) or (objTry < objRef):
            self.atTry = atTry
            self.objTry = objTry
            self.xtTry = xt
        return objTry

    # -- the trial steps as one CUDA graph --------------------------------------------------
    def _trial_body(self):
        """For every step size of g["eps"]: atTry = at - eps dir, its shot and its
        data-term value, on static buffers (one cluster per step size when the
        problem is small, so a batch costs about what one trial step does)."""
        g = self._graph
        out = g["out_buf"]   # [deformation energies, raw data terms] (2, B): written in place
        # the step sizes come from, and the values go to, pinned host buffers: the
        # two copies are part of the replay
        g["eps"].copy_(g["eps_host"], non_blocking=True)
        _, xt, _ = evol.shoot_along_batch(self.x0, g["at"], g["dir"], g["eps"], self.param.KparDiff,
                                          regweight=self.regweight, at_try=g["atTry"], xt=g["xt"],
                                          energy=out[0])
        _dt.value_batch(self.param.errorType, xt[:, -1], self._dshape, self._tc, self._tv, self._Kval,
                        energy_out=out[1])
        g["out_host"].copy_(out, non_blocking=True)
        return out

    def expectTrials(self, dir, steps):
        """Optional line-search hint: the step sizes `steps` along `dir` that the
        next updateTry calls may ask for besides the halving and growth ladders
        (cg's tiny-step probe).  Changes no value, only what a batch holds."""
        self._hint = (dir.diff, [float(e) for e in steps])

    # halving steps of a batch, and the halving depths (counted from the first
    # trial of an iteration) whose growth steps it also holds: cg restarts each
    # iteration at 100 times the last accepted step, so the search returns to
    # that scale after about log2(100) ~ 7 halvings and grows from there
    _LADDER_HALVINGS = 12
    _LADDER_GROWTH_DEPTHS = (5, 6, 7, 8, 9, 10, 11, 4)

    def _trial_ladder(self, eps, cache, dir_diff):
        """The step sizes to evaluate with `eps`: the ones cg may try next from
        it (conjugateGradient.py:140-183), computed with cg's own operations so
        that they compare equal.  When eps is a growth step of an evaluated
        size: eps 1.25^j (chained).  Otherwise eps / 2^k (the halving loops),
        the hinted steps of this direction (cg's tiny-step probe), then the
        first growth steps 1.25 h, 1.25 (1.25 h) of the likely accepted
        halvings h, while the batch has room."""
        B = self._graph["B"]
        if B == 1:
            return [eps]
        if any(1.25 * e == eps for e in cache):
            ladder = [eps]
            while len(ladder) < B:
                ladder.append(1.25 * ladder[-1])
            return ladder
        hint = getattr(self, "_hint", None)
        extra = [e for e in hint[1] if e != eps] if hint is not None and hint[0] is dir_diff else []
        halving = [eps]
        while len(halving) < min(self._LADDER_HALVINGS, B - len(extra)):
            halving.append(halving[-1] / 2)
        ladder = halving + [e for e in extra if e not in halving]
        depth = 1 if B < 24 else 2
        for k in self._LADDER_GROWTH_DEPTHS:
            if k >= len(halving):
                continue
            g = halving[k]
            for _ in range(depth):
                g = 1.25 * g
                if len(ladder) < B and g not in ladder:
                    ladder.append(g)
        h = halving[-1]
        while len(ladder) < B:     # deeper halvings fill what is left
            h = h / 2
            if h not in ladder:
                ladder.append(h)
        return ladder[:B]

    def _graph_update_try(self, dir, eps, objRef):
        """updateTry with the trial steps replayed from a CUDA graph captured on
        the first call: the same kernels on the same inputs (bit-identical to
        the eager path), one launch and one read-back per batch of step sizes.
        A batch evaluates the step sizes the line search asks for next along the
        same direction; later calls for them are answered from it until the
        momenta or the direction change.  The static copies of `at` and of the
        direction are refreshed only when cg hands over new tensors."""
        g = self._graph
        if g is None:
            dev = self.x0.device
            B = evol.trial_batch_size(self.npt, self.dim, self._dshape.cells.shape[0], self._tc.shape[0],
                                      self.param.KparDiff.precision, self._Kval.precision)
            T, n, d = self.at.shape
            g = self._graph = {"B": B, "at": self.at.clone(), "dir": dir.diff.clone(),
                               "eps": torch.full((B,), float(eps), dtype=torch.float64, device=dev),
                               "atTry": torch.empty((B, T, n, d), dtype=torch.float64, device=dev),
                               "xt": torch.empty((B, T + 1, n, d), dtype=torch.float64, device=dev),
                               "out_buf": torch.empty((2, B), dtype=torch.float64, device=dev),
                               "eps_host": torch.full((B,), float(eps), dtype=torch.float64).pin_memory(),
                               "out_host": torch.empty((2, B), dtype=torch.float64).pin_memory(),
                               "at_src": self.at, "dir_src": dir.diff, "cache": {}}
            g["eps_np"], g["out_np"] = g["eps_host"].numpy(), g["out_host"].numpy()
            # capture on a side stream with the low-level calls (the torch.cuda.graph
            # context manager also collects garbage and empties the allocator cache)
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            graph = torch.cuda.CUDAGraph()
            with _gc_paused(), torch.cuda.stream(side):
                with workspace.scope(self):
                    self._trial_body()      # sizes the private workspaces, initialises lazily created state
                with workspace.scope(self):
                    graph.capture_begin()
                    try:
                        self._trial_body()
                    finally:
                        graph.capture_end()
            torch.cuda.current_stream().wait_stream(side)
            g["graph"] = graph
        if g["at_src"] is not self.at:
            g["at"].copy_(self.at)
            g["at_src"] = self.at
            g["cache"] = {}
        if g["dir_src"] is not dir.diff:
            g["dir"].copy_(dir.diff)
            g["dir_src"] = dir.diff
            g["cache"] = {}
        cache = g["cache"]
        eps = float(eps)
        if eps not in cache:
            self._materialize_try()     # the slots are about to be overwritten
            ladder = self._trial_ladder(eps, cache, dir.diff)
            g["eps_np"][:] = ladder
            g["graph"].replay()
            self.calls["trial_batches"] = self.calls.get("trial_batches", 0) + 1
            torch.cuda.current_stream().synchronize()
            ereg, raw = g["out_np"].tolist()
            # the ladder's step sizes are distinct
            cache = g["cache"] = dict(zip(ladder, zip(range(len(ladder)), ereg, raw)))
        b, ereg, raw = cache[eps]
        objTry = self._combine(ereg, raw)
        if self._auto:
            objTry = _Value(objTry, self, ereg, g["xt"][b, -1].clone(), value_bound(self, self._noise, self.obj0))
        if np.isnan(objTry):
            logging.info('Warning: nan in updateTry')
            return 1e500
        if (objRef is None) or (objTry < objRef):
            self._pending_try = (g, b)
            self.objTry = objTry
        return objTry

    def getGradient(self, coeff=1.0):
        """(surfaceMatching.py:301-327): grd.diff = (2 rw a - p_{t+1}) / (coeff T)."""
        self.calls["getGradient"] += 1
        grd = Direction()
        if (self.cudaGraphs and self._fast_data and self.npt <= 2048
                and type(self).endPointGradient is DeviceMatching.endPointGradient):
            grd.diff = self._graph_gradient(float(coeff))
        else:
            px1 = -self.endPointGradient()
            _, dat = evol.covector(self.xt, self.at, px1, self.param.KparDiff, self.regweight, with_dat=True)
            grd.diff = dat / (coeff * self.Tsize)
        grd.aff = np.zeros(self.Afft.shape)
        return grd

    def _gradient_body(self, xt, at, coeff):
        px1 = -self._end_point_gradient(xt[-1])
        _, dat = evol.covector(xt, at, px1, self.param.KparDiff, self.regweight, with_dat=True)
        return dat / (coeff * self.Tsize)

    def _gradient_graph_body(self, g, coeff):
        """The gradient, and the two metric products cg asks for next,
        <g, g> and <g, g_prev> (dotProduct's kernel on the same inputs), into
        pinned host memory; g_prev is the previous gradient of this graph."""
        dat = self._gradient_body(g["xt"], g["at"], coeff)
        if g["dots"]:
            d = evol.metric_dots(g["xt"], dat, [dat, g["prev"]], self.param.KparDiff)
            g["dots_host"].copy_(d, non_blocking=True)
            g["prev"].copy_(dat)
        return dat

    def _graph_gradient(self, coeff):
        """The data-term gradient, the adjoint and the scaling replayed from a CUDA
        graph (the same kernels on copies of xt and at: bit-identical to the
        eager path); a small problem's dozen launches become one.  With the FP32c
        metric products the replay also forms <g, g> and <g, g_prev>, which
        dotProduct then returns for cg's dot(grd, [grd, grdOld])."""
        g = self._grad_graph
        if g is None or g["coeff"] != coeff:
            import types
            K = self.param.KparDiff
            g = self._grad_graph = {"coeff": coeff, "xt": self.xt.clone(), "at": self.at.clone(),
                                    "xt_src": self.xt, "at_src": self.at, "owner": types.SimpleNamespace(),
                                    "dots": K.precision == 'fp32c' and self.npt <= 2048,
                                    "prev": torch.zeros_like(self.at),
                                    "dots_host": torch.zeros(2, dtype=torch.float64).pin_memory(),
                                    "last": None, "last_prev": None}
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            graph = torch.cuda.CUDAGraph()
            with _gc_paused(), torch.cuda.stream(side):
                with workspace.scope(g["owner"]):
                    self._gradient_graph_body(g, coeff)
                with workspace.scope(g["owner"]):
                    graph.capture_begin()
                    try:
                        g["dat"] = self._gradient_graph_body(g, coeff)
                    finally:
                        graph.capture_end()
            torch.cuda.current_stream().wait_stream(side)
            g["graph"] = graph
            g["prev_valid"] = False   # the warm-up call left a gradient in "prev"
        if g["xt_src"] is not self.xt:
            g["xt"].copy_(self.xt)
            g["xt_src"] = self.xt
        if g["at_src"] is not self.at:
            g["at"].copy_(self.at)
            g["at_src"] = self.at
        g["graph"].replay()
        out = g["dat"].clone()
        # the products of this replay: <out, out> and, if the previous gradient
        # of this graph is known, <out, previous>
        g["last_prev"] = g["last"] if g["prev_valid"] else None
        g["last"], g["prev_valid"] = out, True
        g["dots_xt"] = self.xt
        return out

    def _precomputed_dots(self, g1, g2):
        """dotProduct's values from the last gradient replay, when the call is
        dot(g, [g or g_prev, ...]) on that gradient g (g_prev: the previous
        gradient or a copyDir of it) and the trajectory has not changed."""
        g = self._grad_graph
        if g is None or not g["dots"] or g["last"] is None or g1.diff is not g["last"]:
            return None
        if g.get("dots_xt") is not self.xt:
            return None
        idx = []
        for gr in g2:
            src = gr.diff if gr.diff is g["last"] else getattr(gr, "copied_from", None)
            if gr.diff is g["last"]:
                idx.append(0)
            elif g["last_prev"] is not None and (gr.diff is g["last_prev"] or src is g["last_prev"]):
                idx.append(1)
            else:
                return None
        torch.cuda.current_stream().synchronize()
        vals = g["dots_host"].numpy()
        return np.array([vals[i] for i in idx])

    def addProd(self, dir1, dir2, beta):
        d = Direction()
        d.diff = dir1.diff + beta * dir2.diff
        d.aff = dir1.aff
        return d

    def copyDir(self, dir0):
        d = Direction()
        d.diff = dir0.diff.clone()
        d.aff = np.copy(dir0.aff)
        d.copied_from = dir0.diff   # lets dotProduct recognise cg's grdOld
        return d

    def randomDir(self):
        d = Direction()
        d.diff = torch.randn((self.Tsize, self.npt, self.dim), dtype=torch.float64, device=self.x0.device)
        d.aff = np.zeros(self.Afft.shape)
        return d

    def dotProduct(self, g1, g2):
        """sum_t <g2_t, K(x_t) g1_t> (surfaceMatching.py:353-377), FP64 on the device."""
        self.calls["dotProduct"] += 1
        K = self.param.KparDiff
        pre = self._precomputed_dots(g1, g2)
        if pre is not None:
            return pre
        if K.precision == 'fp32c' and self.npt <= 2048 and 1 <= len(g2) <= 8:
            # all T steps and directions in two launches (pointEvolution.metric_dots)
            return evol.metric_dots(self.xt, g1.diff, [gr.diff for gr in g2], K).cpu().numpy()
        if K.precision == 'fp32c':
            # the T applyK sums as one ragged launch (one segment per time step)
            T, N, d = self.Tsize, self.npt, self.dim
            U = _rg.applyk_segments(self.xt[:T].reshape(-1, d), to_dev(g1.diff).reshape(-1, d),
                                    [t * N for t in range(T)], [N] * T, [K.sigma] * T, _rg.kernel_order(K))
            G2 = torch.stack([to_dev(gr.diff).reshape(-1) for gr in g2])
            return (G2 @ U.reshape(-1)).cpu().numpy()
        acc = torch.zeros(len(g2), dtype=torch.float64, device=self.x0.device)
        for t in range(self.Tsize):
            u = K.applyK(self.xt[t], g1.diff[t])
            for ll, gr in enumerate(g2):
                acc[ll] += (gr.diff[t] * u).sum()
        return acc.cpu().numpy()

    def acceptVarTry(self):
        self.obj = self.objTry
        pend = self._pending_try
        if pend is not None:
            # one copy out of the batch slot (the eager path's atTry.clone())
            g, b = pend
            self._pending_try = None
            self.at = g["atTry"][b].clone()
            self.xt = g["xt"][b].clone()
            self.__dict__["_atTry"] = self.at
            self.__dict__["_xtTry"] = self.xt
            return
        self.at = self.atTry.clone()
        if self.xtTry is not None:
            self.xt = self.xtTry

    def endOfIteration(self):
        self.iter += 1
        self.fvDef.updateVertices(self.xt[-1])

    def endOptim(self):
        if isinstance(self.obj, _Value):
            self.obj = float(self.obj.refine())
