"""Model-fitting action log-likelihood (``pymdp_b200.fitting``) against the
FP64 oracle of ``pymdp/likelihoods.py:7-45``: the value per subject, and its
gradient w.r.t. A/B logits, C and log gamma against central finite
differences (h = 1e-3, FP64) on a parameter subsample. The model is the
fitting workload's (S=[8,4], O=[8,4,3] on both factors, U=[4,1], policy_len 2,
num_iter 16) with a few subjects and trials."""

import numpy as np
import pytest
import torch

from oracle import fitting as ofit

pytestmark = pytest.mark.gpu

H = 1e-3
GRAD_REL = 1e-4
LL_REL = 1e-5


def _setup(n, T, seed):
    from pymdp_b200.fitting import FitModel
    fm = FitModel([8, 4], [8, 4, 3], [4, 1], policy_len=2, num_iter=16)
    g = torch.Generator(device="cuda").manual_seed(seed)
    A, B, C, lg = fm.init_params(n, g)
    obs, acts = fm.simulate(A, B, C, lg, T, g)
    return fm, A, B, C, lg, obs, acts


def _np(params):
    A, B, C, lg = params
    f = lambda xs: [x.detach().double().cpu().numpy() for x in xs]
    return f(A), f(B), f(C), lg.detach().double().cpu().numpy()


@pytest.mark.parametrize("form", ["log", "probs_as_logits"])
def test_fit_log_likelihood_matches_oracle(form):
    fm, A, B, C, lg, obs, acts = _setup(4, 5, 11)
    ll = fm.log_likelihood(A, B, C, lg, obs, acts, form=form, per_subject=True)
    An, Bn, Cn, lgn = _np((A, B, C, lg))
    o, a = obs.cpu().numpy(), acts.cpu().numpy()
    for n in range(4):
        ref = ofit.subject_log_likelihood([x[n] for x in An], [x[n] for x in Bn], [x[n] for x in Cn], lgn[n],
                                          o[:, n], a[:, n], fm.U, fm.policy_len, fm.A_dependencies, fm.num_iter,
                                          form=form)
        assert abs(float(ll[n]) - ref) <= LL_REL * max(abs(ref), 1.0), (n, float(ll[n]), ref)


@pytest.mark.parametrize("form", ["log", "probs_as_logits"])
def test_fit_gradient_matches_finite_differences(form):
    n, T = 2, 4
    fm, A, B, C, lg, obs, acts = _setup(n, T, 3)
    params = [x.clone().requires_grad_(True) for x in A + B + C + [lg]]
    nA, nB, nC = len(A), len(B), len(C)
    Ap, Bp, Cp, lgp = params[:nA], params[nA:nA + nB], params[nA + nB:nA + nB + nC], params[-1]
    fm.log_likelihood(Ap, Bp, Cp, lgp, obs, acts, form=form).backward()
    base = [x.detach().double().cpu().numpy() for x in params]
    o = obs.cpu().numpy().transpose(1, 0, 2)
    a = acts.cpu().numpy().transpose(1, 0, 2)

    def f(vals):
        return ofit.log_likelihood(vals[:nA], vals[nA:nA + nB], vals[nA + nB:nA + nB + nC], vals[-1], o, a, fm.U,
                                   fm.policy_len, fm.A_dependencies, fm.num_iter, form=form)

    rng = np.random.default_rng(0)
    gmax = max(float(p.grad.abs().max()) for p in params)
    worst = 0.0
    for i, arr in enumerate(base):
        picks = [tuple(int(rng.integers(0, s)) for s in arr.shape) for _ in range(4 if arr.ndim > 1 else n)]
        if arr.ndim == 1:
            picks = [(j,) for j in range(n)]
        for key in picks:
            vp = [x.copy() for x in base]; vp[i][key] += H
            vm = [x.copy() for x in base]; vm[i][key] -= H
            fd = (f(vp) - f(vm)) / (2 * H)
            got = float(params[i].grad[key])
            err = abs(got - fd) / max(abs(fd), 1e-2 * gmax)
            worst = max(worst, err)
            assert err <= GRAD_REL, (i, key, got, fd, err)
    print(f"max relative gradient error ({form}): {worst:.2e}")


def test_graphed_log_likelihood_matches_eager():
    """The CUDA-graph replay of forward + backward gives the eager value and
    gradients, and follows in-place parameter updates."""
    from pymdp_b200.fitting import GraphedLogLikelihood
    fm, A, B, C, lg, obs, acts = _setup(8, 6, 5)
    params = [x.clone().requires_grad_(True) for x in A + B + C + [lg]]
    split = lambda ps: (ps[:3], ps[3:5], ps[5:8], ps[8])  # noqa: E731
    ll = fm.log_likelihood(*split(params), obs, acts)
    ll.backward()
    ref = float(ll.detach())
    gref = [p.grad.clone() for p in params]
    del ll
    for p in params:
        p.grad = None
    graphed = GraphedLogLikelihood(fm, params, obs, acts)
    assert abs(float(graphed()) - ref) <= LL_REL * abs(ref)
    for p, g in zip(params, gref):
        torch.testing.assert_close(p.grad, g, rtol=1e-5, atol=1e-6)
    with torch.no_grad():
        params[-1].add_(0.1)
        ref2 = float(fm.log_likelihood(*split(params), obs, acts))
    assert abs(float(graphed()) - ref2) <= LL_REL * abs(ref2)
