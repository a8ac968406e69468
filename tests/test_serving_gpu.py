"""Ragged launches and the continuous-batching server on the GPU.

* each lddmm_ragged_* entry point against the single-problem entry points,
  request by request (FP32c: 1e-6 of the row scale; FP64: 1e-12);
* each request's ragged result is bit-identical alone and in a mix of
  requests of other sizes and kernel widths;
* the server: every result is bit-identical alone and in the mix (also when
  requests arrive late or the HBM budget admits one at a time), and it agrees
  with the single-problem SurfaceMatching driver.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _shape(subdiv, keep, seed, bumps=6):
    from registration_b200 import geometry as geo
    rng = np.random.default_rng(seed)
    v, f = geo.icosphere(subdiv)
    if keep < len(v):
        v, f = geo.decimate(v, f, keep, rng)
    vt = geo.bumped_sphere(v, f, bumps, 0.3, 0.15, rng)
    return v, f, vt


SHAPES = [(2, 162, 1), (2, 120, 2), (3, 400, 3), (2, 90, 4)]
SIGMAS = [0.3, 0.45, 0.25, 0.35]


def _i64(a):
    return (ctypes.c_int64 * len(a))(*[int(x) for x in a])


def _f64(a):
    return (ctypes.c_double * len(a))(*[float(x) for x in a])


def _ragged_shoot(x0s, ats, sigmas, rws, order=10):
    from registration_b200 import _lib
    from registration_b200.device import ptr, stream_handle, workspace
    T, d = ats[0].shape[0], x0s[0].shape[1]
    v_off = np.concatenate([[0], np.cumsum([len(x) for x in x0s])])
    X0 = torch.cat(x0s)
    AT = torch.cat([a.reshape(-1, d) for a in ats])
    XT = torch.empty(((T + 1) * int(v_off[-1]), d), dtype=torch.float64, device="cuda")
    E = torch.empty(len(x0s), dtype=torch.float64, device="cuda")
    wsb = _lib.query("lddmm_ragged_shoot_f32c_workspace", len(x0s), _i64(v_off), d, T, order)
    ws = workspace.get(wsb)
    _lib.call("lddmm_ragged_shoot_f32c", len(x0s), _i64(v_off), d, ptr(X0), ptr(AT), T, _f64(sigmas), order,
              _f64(rws), ptr(XT), ptr(E), ptr(ws), wsb, stream_handle())
    xts = [XT[(T + 1) * v_off[i]:(T + 1) * v_off[i + 1]].view(T + 1, -1, d) for i in range(len(x0s))]
    return xts, E


def _ragged_cov(xts, ats, px1s, sigmas, rws, order=10):
    from registration_b200 import _lib
    from registration_b200.device import ptr, stream_handle, workspace
    T, d = ats[0].shape[0], xts[0].shape[2]
    v_off = np.concatenate([[0], np.cumsum([x.shape[1] for x in xts])])
    XT = torch.cat([x.reshape(-1, d) for x in xts])
    AT = torch.cat([a.reshape(-1, d) for a in ats])
    PX = torch.cat(px1s)
    PXT = torch.empty_like(XT)
    DAT = torch.empty_like(AT)
    wsb = _lib.query("lddmm_ragged_covector_f32c_workspace", len(xts), _i64(v_off), d, T, order)
    ws = workspace.get(wsb)
    _lib.call("lddmm_ragged_covector_f32c", len(xts), _i64(v_off), d, ptr(XT), ptr(AT), T, ptr(PX), _f64(sigmas),
              order, _f64(rws), ptr(PXT), ptr(DAT), ptr(ws), wsb, stream_handle())
    pxts = [PXT[(T + 1) * v_off[i]:(T + 1) * v_off[i + 1]].view(T + 1, -1, d) for i in range(len(xts))]
    dats = [DAT[T * v_off[i]:T * v_off[i + 1]].view(T, -1, d) for i in range(len(xts))]
    return pxts, dats


def _ragged_applyk(xs, ys, betas, sigmas, order):
    from registration_b200 import _lib
    from registration_b200.device import ptr, stream_handle, workspace
    d, dimb = xs[0].shape[1], betas[0].shape[1]
    X, Y, B = torch.cat(xs), torch.cat(ys), torch.cat(betas)
    tc = [len(x) for x in xs]
    sc = [len(y) for y in ys]
    ts = np.concatenate([[0], np.cumsum(tc)])[:-1]
    ss = np.concatenate([[0], np.cumsum(sc)])[:-1]
    F = torch.empty((sum(tc), dimb), dtype=torch.float64, device="cuda")
    wsb = _lib.query("lddmm_ragged_applyk_f32c_workspace", len(xs), _i64(tc), _i64(sc), d, dimb, order)
    ws = workspace.get(wsb)
    _lib.call("lddmm_ragged_applyk_f32c", len(xs), _i64(ts), _i64(tc), _i64(ss), _i64(sc), d, ptr(X), ptr(Y),
              ptr(B), dimb, _f64(sigmas), order, ptr(F), ptr(ws), wsb, stream_handle())
    off = np.concatenate([[0], np.cumsum(tc)])
    return [F[off[i]:off[i + 1]] for i in range(len(xs))]


def _ragged_data(norm, shapes, verts, tcs, tvs, sigmas, precision, energy=True, grad=False, order=10, frame=None):
    from registration_b200 import _dataterm as _dt
    from registration_b200 import _lib
    from registration_b200.device import ptr, stream_handle, workspace
    k = shapes[0].cells.shape[1]
    d = verts[0].shape[1]
    v_off, c_off, c2_off = [0], [0], [0]
    cells, vptr, vidx = [], [], []
    for shp, v, tc in zip(shapes, verts, tcs):
        cells.append(shp.cells + v_off[-1])
        vptr.append(shp.vptr[:-1] + c_off[-1] * k)
        vidx.append(shp.vidx + c_off[-1] * k)
        v_off.append(v_off[-1] + len(v))
        c_off.append(c_off[-1] + shp.cells.shape[0])
        c2_off.append(c2_off[-1] + (0 if tc is None else len(tc)))
    V = torch.cat(verts)
    C = torch.cat(cells)
    VP = torch.cat(vptr + [torch.full((1,), c_off[-1] * k, dtype=torch.int64, device="cuda")])
    VI = torch.cat(vidx)
    has_t = tcs[0] is not None
    C2 = torch.cat(tcs) if has_t else None
    S2 = torch.cat(tvs) if has_t else None
    n = len(shapes)
    E = torch.empty(n, dtype=torch.float64, device="cuda") if energy else None
    PX = torch.empty_like(V) if grad else None
    sfx = "f32c" if precision == "fp32c" else "f64"
    nid = _dt.NORMS[norm]
    wsb = _lib.query("lddmm_ragged_dataterm_%s_workspace" % sfx, n, k, nid, _i64(v_off), _i64(c_off), _i64(c2_off),
                     d, order, int(energy), int(grad))
    ws = workspace.get(wsb)
    _lib.call("lddmm_ragged_dataterm_" + sfx, n, k, nid, _i64(v_off), _i64(c_off), _i64(c2_off), ptr(V), d, ptr(C),
              ptr(C2) if has_t else None, ptr(S2) if has_t else None, _f64(sigmas), order, 1e-10, 1e-10, frame,
              ptr(E) if energy else None, ptr(VP), ptr(VI), ptr(PX) if grad else None, ptr(ws), wsb,
              stream_handle())
    pxs = [PX[v_off[i]:v_off[i + 1]] for i in range(n)] if grad else None
    return E, pxs


def _close(a, b, tol):
    return float((a - b).abs().max()) <= tol * max(float(b.abs().max()), 1e-300)


@pytest.fixture(scope="module")
def problems():
    from registration_b200 import _dataterm as _dt
    out = []
    for i, (sub, keep, seed) in enumerate(SHAPES):
        v, f, vt = _shape(sub, keep, seed)
        rng = np.random.default_rng(100 + i)
        T = 5
        at = torch.from_numpy(0.05 * rng.standard_normal((T, len(v), 3))).cuda()
        c2, s2 = _dt.cell_geometry(vt, f)
        out.append(dict(v=torch.from_numpy(v).cuda(), f=f, vt=vt, at=at, sigma=SIGMAS[i], rw=0.5 + 0.25 * i,
                        shape=_dt.DeviceShape(f, len(v)), tshape=_dt.DeviceShape(f, len(vt)),
                        tc=torch.from_numpy(c2).cuda(), tv=torch.from_numpy(s2).cuda(),
                        px1=torch.from_numpy(rng.standard_normal((len(v), 3))).cuda()))
    return out


def test_ragged_shoot_and_covector_match_single(problems):
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import pointEvolution as evol
    xts, E = _ragged_shoot([p["v"] for p in problems], [p["at"] for p in problems], [p["sigma"] for p in problems],
                           [p["rw"] for p in problems])
    pxts, dats = _ragged_cov(xts, [p["at"] for p in problems], [p["px1"] for p in problems],
                             [p["sigma"] for p in problems], [p["rw"] for p in problems])
    for i, p in enumerate(problems):
        K = kf.Kernel(name="gauss", sigma=p["sigma"], precision="fp32c")
        xt, e = evol.shoot(p["v"], p["at"], K, regweight=p["rw"], with_energy=True)
        # FP32c sums in both; the frames and chunkings are the same
        assert _close(xts[i] - p["v"], xt - p["v"], 1e-6)
        assert abs(float(E[i]) - float(e)) <= 1e-6 * abs(float(e))
        pxt, dat = evol.covector(xt, p["at"], p["px1"], K, p["rw"], with_dat=True)
        assert _close(pxts[i], pxt, 1e-6) and _close(dats[i], dat, 1e-6)


def test_ragged_shoot_alone_equals_mix(problems):
    args = lambda ps: ([p["v"] for p in ps], [p["at"] for p in ps], [p["sigma"] for p in ps], [p["rw"] for p in ps])
    xts, E = _ragged_shoot(*args(problems))
    pxts, dats = _ragged_cov(xts, [p["at"] for p in problems], [p["px1"] for p in problems],
                             [p["sigma"] for p in problems], [p["rw"] for p in problems])
    for i, p in enumerate(problems):
        xa, Ea = _ragged_shoot(*args([p]))
        assert torch.equal(xa[0], xts[i]) and float(Ea[0]) == float(E[i])
        pa, da = _ragged_cov(xa, [p["at"]], [p["px1"]], [p["sigma"]], [p["rw"]])
        assert torch.equal(pa[0], pxts[i]) and torch.equal(da[0], dats[i])
    # a different mix (reversed order, one request left out)
    idx = [3, 2, 1]
    xs, Es = _ragged_shoot(*args([problems[i] for i in idx]))
    for j, i in enumerate(idx):
        assert torch.equal(xs[j], xts[i]) and float(Es[j]) == float(E[i])


@pytest.mark.parametrize("order", [10, 3, 1])
def test_ragged_applyk_matches_single_and_alone(problems, order):
    from registration_b200 import kernelFunctions as kf
    rng = np.random.default_rng(order)
    xs = [p["v"] for p in problems]
    ys = [p["v"][::2].contiguous() for p in problems]
    bs = [torch.from_numpy(rng.standard_normal((len(y), 3))).cuda() for y in ys]
    sig = [p["sigma"] for p in problems]
    fs = _ragged_applyk(xs, ys, bs, sig, order)
    name = "gauss" if order > 4 else "laplacian"
    for i in range(len(xs)):
        K = kf.Kernel(name=name, sigma=sig[i], order=order if order <= 4 else 3, precision="fp32c")
        ref = K.applyK(ys[i], bs[i], firstVar=xs[i])
        assert _close(fs[i], ref, 1e-6)
        alone = _ragged_applyk([xs[i]], [ys[i]], [bs[i]], [sig[i]], order)
        assert torch.equal(alone[0], fs[i])


@pytest.mark.parametrize("norm", ["current", "measure", "varifold"])
@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_ragged_dataterm_matches_single_and_alone(problems, norm, precision):
    from registration_b200 import _dataterm as _dt
    from registration_b200 import kernelFunctions as kf
    verts = [p["v"] + 0.01 for p in problems]
    shapes = [p["shape"] for p in problems]
    tcs, tvs = [p["tc"] for p in problems], [p["tv"] for p in problems]
    sig = [0.5 * p["sigma"] for p in problems]
    E, pxs = _ragged_data(norm, shapes, verts, tcs, tvs, sig, precision, energy=True, grad=True)
    E0, _ = _ragged_data(norm, [p["tshape"] for p in problems],
                         [torch.from_numpy(p["vt"]).cuda() for p in problems], [None] * 4, [None] * 4, sig,
                         precision)
    tol = 1e-12 if precision == "fp64" else 1e-6
    for i, p in enumerate(problems):
        K = kf.Kernel(name="gauss", sigma=sig[i], precision=precision)
        e, px = _dt.dataterm(norm, verts[i], shapes[i], tcs[i], tvs[i], K, energy=True, grad=True)
        # NormDef = <S,S> - 2<S,T> is a difference of large terms: compare on the scale of the self term
        e_self, _ = _dt.dataterm(norm, verts[i], shapes[i], None, None, K, energy=True)
        assert abs(float(E[i]) - float(e)) <= tol * abs(float(e_self))
        assert _close(pxs[i], px, tol if precision == "fp64" else 1e-5)
        e0, _ = _dt.dataterm(norm, torch.from_numpy(p["vt"]).cuda(), p["tshape"], None, None, K, energy=True)
        assert abs(float(E0[i]) - float(e0)) <= tol * abs(float(e0))
        Ea, pa = _ragged_data(norm, [shapes[i]], [verts[i]], [tcs[i]], [tvs[i]], [sig[i]], precision, grad=True)
        assert float(Ea[0]) == float(E[i]) and torch.equal(pa[0], pxs[i])


def _make_requests(idx, iters=8, err="varifold"):
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import serving
    from registration_b200 import surfaces as sf
    from registration_b200.surfaceMatching import SurfaceMatchingParam
    out = []
    for i in idx:
        sub, keep, seed = SHAPES[i]
        v, f, vt = _shape(sub, keep, seed)
        s = SIGMAS[i]
        param = SurfaceMatchingParam(timeStep=0.2, KparDiff=kf.Kernel(name="gauss", sigma=s, precision="fp32c"),
                                     KparDist=kf.Kernel(name="gauss", sigma=s / 2, precision="fp32c"),
                                     sigmaError=0.5, errorType=err)
        out.append(serving.MatchRequest(sf.Surface(FV=[f, v]), sf.Surface(FV=[f, vt]), param, maxIter=iters,
                                        regWeight=1.0, rid=i))
    return out


def _result(req):
    assert req.error is None, req.error
    return req.result


def test_serving_alone_equals_mix():
    from registration_b200 import serving
    mix = _make_requests(range(4))
    eng = serving.serve(mix)
    st = eng.stats()
    assert st["finished"] == 4 and st["failed"] == 0 and st["max_batch"] >= 2
    for r in mix:
        alone = _make_requests([r.rid])
        serving.serve(alone)
        a, b = _result(alone[0]), _result(r)
        assert a["obj"] == b["obj"] and a["iters"] == b["iters"]
        assert torch.equal(a["at"], b["at"])


def test_serving_late_arrivals_and_hbm_budget_are_bit_identical():
    import time
    from registration_b200 import serving
    base = _make_requests(range(4))
    serving.serve(base)
    # staggered arrivals: requests join while others are mid-optimisation
    late = _make_requests(range(4))
    t0 = time.perf_counter()
    for j, r in enumerate(late):
        r.arrival = t0 + 0.002 * j
    eng = serving.serve(late)
    # a budget that holds the largest request and little else
    one = _make_requests(range(4))
    for r in one:
        r.arrival = None
    budget = max(r.hbm_bytes() for r in one) * 1.01
    eng1 = serving.serve(one, hbm_budget_bytes=budget)
    assert eng1.stats()["peak_hbm_bytes"] <= budget and eng1.stats()["max_active"] < 4
    for a, b, c in zip(base, late, one):
        assert _result(a)["obj"] == _result(b)["obj"] == _result(c)["obj"]
        assert torch.equal(_result(a)["at"], _result(b)["at"]) and torch.equal(_result(a)["at"], _result(c)["at"])
        assert b.start >= b.arrival
    assert eng.stats()["max_active"] >= 2


def test_faulty_and_cancelled_requests_fail_alone():
    """A request with a NaN target vertex fails at admission; one whose initial
    momenta overflow FP32 (1e200) gets a non-finite objective on the GPU and
    fails with FloatingPointError; one cancelled after three value rounds ends
    with RequestCancelled.  All three give back their slot and budget, and the
    requests sharing their launches finish bit-identical to their solo runs."""
    from registration_b200 import serving
    from registration_b200 import surfaces as sf

    good = _make_requests([0, 2])
    victim = _make_requests([1])[0]
    base = _make_requests([3])[0]
    vt = base.v1.copy()
    vt[5, 2] = np.nan
    nan_target = serving.MatchRequest(sf.Surface(FV=[base.f0, base.v0]), sf.Surface(FV=[base.f1, vt]), base.param,
                                      maxIter=8, rid="nan-target")
    huge = serving.MatchRequest(sf.Surface(FV=[base.f0, base.v0]), sf.Surface(FV=[base.f1, base.v1]), base.param,
                                maxIter=8, rid="overflow",
                                at_init=np.full((base.T, base.n, 3), 1e200))

    class Cancelling(serving.ServingEngine):
        def _do_value(self, items):
            for p, _ in items:
                if p.req is victim and p.calls["value"] >= 3:
                    victim.cancel()
            return super()._do_value(items)

    eng = Cancelling()
    for r in good + [victim, nan_target, huge]:
        eng.submit(r)
    eng.run()
    assert isinstance(nan_target.error, ValueError) and "not finite" in str(nan_target.error)
    assert isinstance(huge.error, FloatingPointError)
    assert isinstance(victim.error, serving.RequestCancelled)
    st = eng.stats()
    assert st["failed"] == 3 and st["finished"] == 5
    assert eng.n_active == 0 and eng.hbm_in_use == 0
    for r in good:
        alone = _make_requests([r.rid])
        serving.serve(alone)
        a, b = _result(alone[0]), _result(r)
        assert a["obj"] == b["obj"] and a["iters"] == b["iters"] and torch.equal(a["at"], b["at"])


def test_serving_rejects_requests_above_the_budget():
    from registration_b200 import serving
    reqs = _make_requests([0, 2], iters=2)
    eng = serving.serve(reqs, hbm_budget_bytes=reqs[0].hbm_bytes() * 1.01)
    assert reqs[0].error is None
    assert isinstance(reqs[1].error, MemoryError)
    assert eng.stats()["failed"] == 1


def test_serving_matches_single_problem_driver():
    """The same problem through SurfaceMatching (single-problem kernels, FP64
    data-term values in the line search): the served 'auto' line search takes
    the FP64 decisions."""
    from registration_b200 import serving
    from registration_b200 import surfaces as sf
    from registration_b200.surfaceMatching import SurfaceMatching
    reqs = _make_requests([0, 1], iters=10)
    serving.serve(reqs)
    for r in reqs:
        sm = SurfaceMatching(Template=sf.Surface(FV=[r.f0, r.v0]), Target=sf.Surface(FV=[r.f1, r.v1]),
                             param=r.param, maxIter=10, regWeight=1.0, verb=r.verb, testGradient=False,
                             lineSearchPrecision="fp64")
        sm.optimizeMatching()
        res = _result(r)
        # same decisions; shooting and gradients are FP32c sums in both (ragged
        # vs single-problem packing and chunking), so the final objective -- a
        # small difference of norms -- agrees to the FP32c bar, 1e-5 relative
        assert res["iters"] == sm.iter
        assert abs(res["obj"] - sm.obj) <= 1e-5 * abs(sm.obj), (res["obj"], sm.obj)


def test_ragged_call_refused_while_capturing():
    """Ragged entry points copy host-built segment tables to the device on each
    call; on a stream that is capturing a CUDA graph they return an error
    before enqueueing anything (a captured copy would keep a stale host address)."""
    import torch
    from registration_b200 import _ragged as rg
    x = torch.rand(64, 3, dtype=torch.float64, device="cuda")
    a = torch.rand(64, 3, dtype=torch.float64, device="cuda")
    rg.applyk_segments(x, a, [0, 32], [32, 32], [0.3, 0.3], 10)   # eager: fine
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            with pytest.raises(ValueError, match="captured"):
                rg.applyk_segments(x, a, [0, 32], [32, 32], [0.3, 0.3], 10)
        finally:
            g.capture_end()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()


def _curve_requests(idx, iters=8):
    from registration_b200 import curves as cv
    from registration_b200 import geometry as geo
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import serving
    from registration_b200.curveMatching import CurveMatchingParam
    out = []
    for i in idx:
        rng = np.random.default_rng(40 + i)
        v, _ = geo.ellipse_curve(64 + 32 * i, 1.0, 0.6)
        vt, _ = geo.bumped_curve(v, 3, 0.3, 0.1, rng)
        param = CurveMatchingParam(timeStep=0.1, KparDiff=kf.Kernel(name="gauss", sigma=0.5),
                                   KparDist=kf.Kernel(name="gauss", sigma=0.5), sigmaError=0.2,
                                   errorType="current")
        out.append(serving.MatchRequest(cv.Curve(pointSet=v), cv.Curve(pointSet=vt), param, maxIter=iters, rid=i))
    return out


def test_served_curves_alone_equal_mix_and_match_curve_matching():
    """Curve requests (edges, d = 2) follow CurveMatching's protocol (cg's
    first step 10): alone == in the mix bit for bit, and the same decisions as
    the single-problem CurveMatching with FP64 line-search values.  The single
    problem's FP32c kernel sums run in other kernels (single-launch ones for
    these sizes) than the served ragged launches, so the final energies agree
    to the FP32c scale of the objective, 1e-5 of obj0."""
    from registration_b200 import curves as cv
    from registration_b200 import serving
    from registration_b200.curveMatching import CurveMatching
    mix = _curve_requests(range(3))
    serving.serve(mix, line_search_precision="fp64")
    for r in mix:
        alone = _curve_requests([r.rid])
        serving.serve(alone, line_search_precision="fp64")
        a, b = _result(alone[0]), _result(r)
        assert a["obj"] == b["obj"] and torch.equal(a["at"], b["at"])
        cm = CurveMatching(Template=cv.Curve(pointSet=r.v0), Target=cv.Curve(pointSet=r.v1), param=r.param,
                           maxIter=8, saveRate=0, lineSearchPrecision="fp64")
        cm.optimizeMatching()
        assert b["iters"] == cm.iter
        assert abs(b["obj"] - cm.obj) <= 1e-5 * abs(cm.obj0), (b["obj"], cm.obj, cm.obj0)
