"""The hand-written backward of the shooting + data-term objective.

* central finite differences in FP64 along random directions (a and x0);
* the reference's landmarkHamiltonianGradient (oracle): dE/da_t = dt K(x_t) dat_t;
* checkpointed recompute gives the gradient of the stored trajectory (each
  segment is packed in its own centred frame, so the agreement is to rounding:
  1e-12 relative in FP64, 1e-6 in FP32c).
Tolerances are written at each assertion.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problem(precision, subdiv=2, T=5, seed=0, err="current", sig_diff=0.4, sig_dist=0.3):
    from registration_b200 import autograd as ag
    from registration_b200 import geometry as geo
    from registration_b200 import kernelFunctions as kf
    from registration_b200 import surfaces as sf
    rng = np.random.default_rng(seed)
    v, f = geo.icosphere(subdiv)
    vt = geo.bumped_sphere(v, f, 6, 0.3, 0.15, rng)
    tmpl, tgt = sf.Surface(FV=[f, v]), sf.Surface(FV=[f, vt])
    geom = ag.Geometry(tmpl, tgt, kf.Kernel(name="gauss", sigma=sig_diff, precision=precision),
                       kf.Kernel(name="gauss", sigma=sig_dist, precision=precision), err, sigmaError=0.5,
                       regweight=0.8)
    at = torch.from_numpy(0.02 * rng.standard_normal((T, len(v), 3))).cuda()
    x0 = torch.from_numpy(v).cuda()
    return geom, at, x0, (v, f, vt), rng


@pytest.mark.parametrize("err", ["current", "varifold"])
def test_gradient_matches_central_differences_fp64(err):
    from registration_b200 import autograd as ag
    geom, at, x0, _, rng = _problem("fp64", err=err)
    a = at.clone().requires_grad_(True)
    x = x0.clone().requires_grad_(True)
    E = ag.lddmm_objective(a, x, geom)
    E.backward()
    for which in ("a", "x0"):
        base = at if which == "a" else x0
        grad = a.grad if which == "a" else x.grad
        d = torch.from_numpy(rng.standard_normal(tuple(base.shape))).cuda()
        h = 1e-4
        if which == "a":
            ep = float(ag.lddmm_objective(at + h * d, x0, geom))
            em = float(ag.lddmm_objective(at - h * d, x0, geom))
        else:
            ep = float(ag.lddmm_objective(at, x0 + h * d, geom))
            em = float(ag.lddmm_objective(at, x0 - h * d, geom))
        fd = (ep - em) / (2 * h)
        an = float((grad * d).sum())
        # central differences: O(h^2) truncation, FP64 evaluation
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-12), (which, fd, an)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32c", 1e-5)])
def test_gradient_matches_reference_hamiltonian_gradient(oracle_lib, precision, tol):
    """dE/da_t = dt K(x_t) dat_t with dat from the reference's landmarkHamiltonianGradient."""
    from oracle import lddmm_ref as ref
    from registration_b200 import autograd as ag
    geom, at, x0, (v, f, vt), _ = _problem(precision)
    a = at.clone().requires_grad_(True)
    ag.lddmm_objective(a, x0, geom).backward()
    KR = ref.Kernel(name="gauss", sigma=0.4)
    KD = ref.Kernel(name="gauss", sigma=0.3)
    at_np = at.cpu().numpy()
    T = at_np.shape[0]
    xt = ref.landmarkDirectEvolutionEuler(v, at_np, KR)
    fvD, fv1 = ref.Surface(FV=[f, xt[-1]]), ref.Surface(FV=[f, vt])
    px1 = -ref.currentNormGradient(fvD, fv1, KD) / 0.5 ** 2
    dat, _ = ref.landmarkHamiltonianGradient(v, at_np, px1, KR, 0.8)
    expect = np.stack([(1.0 / T) * KR.applyK(xt[t], dat[t]) for t in range(T)])
    got = a.grad.cpu().numpy()
    assert np.abs(got - expect).max() <= tol * np.abs(expect).max()


def _close(a, b, tol):
    return float((a - b).abs().max()) <= tol * float(b.abs().max())


@pytest.mark.parametrize("precision,tol", [("fp32c", 1e-6), ("fp64", 1e-12)])
def test_checkpointed_backward_equals_stored_trajectory(precision, tol):
    from registration_b200 import autograd as ag
    geom, at, x0, _, _ = _problem(precision, T=7)
    grads = []
    for c in (None, 2, 3):
        a = at.clone().requires_grad_(True)
        x = x0.clone().requires_grad_(True)
        E = ag.lddmm_objective(a, x, geom, checkpoint_every=c)
        E.backward()
        grads.append((float(E), a.grad.clone(), x.grad.clone()))
    for e, ga, gx in grads[1:]:
        assert abs(e - grads[0][0]) <= tol * abs(grads[0][0])
        assert _close(ga, grads[0][1], tol) and _close(gx, grads[0][2], tol)
    # the recomputed segments equal the forward's own segments exactly: the
    # same call twice gives bit-identical gradients
    a = at.clone().requires_grad_(True)
    ag.lddmm_objective(a, x0, geom, checkpoint_every=2).backward()
    assert torch.equal(a.grad, grads[1][1])


def test_memory_budget_switches_to_checkpoints():
    from registration_b200 import autograd as ag
    geom, at, x0, _, _ = _problem("fp32c", T=9)
    a1 = at.clone().requires_grad_(True)
    ag.lddmm_objective(a1, x0, geom).backward()
    a2 = at.clone().requires_grad_(True)
    ag.lddmm_objective(a2, x0, geom, memory_budget_bytes=1024).backward()   # forces sqrt(T) segments
    assert _close(a2.grad, a1.grad, 1e-6)
