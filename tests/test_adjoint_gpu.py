"""Adjoint kernels (b2_fpi_obs_bwd, b2_neg_efe_bwd through
pymdp_b200.autograd) against central finite differences of the FP64 oracle.

The reference obtains these gradients with jax.grad of its JAX path
(pymdp/ffi/_core.py:282-310); here the reverse passes are native. Losses are
random linear functionals of the outputs; each gradient entry is checked on a
sample of inputs with h = 1e-6 central differences in FP64. Tolerance: 1e-4
relative to the gradient's scale (FPI adjoint is FP64 on chip; the EFE adjoint
accumulates in FP32)."""

import numpy as np
import pytest
import torch

from oracle import efe as oefe
from oracle import fpi as ofpi

pytestmark = pytest.mark.gpu

H = 1e-6
REL = 1e-4


def cuda(x):
    return torch.as_tensor(np.asarray(x), device="cuda").float()


def _dir(rng, shape, alpha=1.0):
    g = rng.gamma(alpha, size=shape) + 1e-3
    return (g / g.sum(1, keepdims=True)).astype(np.float32)


@pytest.mark.parametrize("case", [
    dict(S=[3, 4], O=[3, 2], deps=[[0, 1], [1]], num_iter=8),
    dict(S=[2, 3, 2], O=[4, 3], deps=[[0, 1, 2], [2, 0]], num_iter=5),
])
def test_fpi_adjoint_matches_finite_differences(case):
    from pymdp_b200 import ffi
    from pymdp_b200.autograd import FpiObs
    S, O, deps, n = case["S"], case["O"], case["deps"], case["num_iter"]
    rng = np.random.default_rng(5)
    batch = 2
    A = [_dir(rng, (batch, O[m]) + tuple(S[d] for d in deps[m])) for m in range(len(O))]
    prior = [_dir(rng, (batch, s)) for s in S]
    obs = rng.integers(0, np.array(O), size=(batch, len(O))).astype(np.int32)
    r = rng.normal(size=(batch, sum(S)))
    A_t = [cuda(a).requires_grad_(True) for a in A]
    p_t = [cuda(p).requires_grad_(True) for p in prior]
    A_flat, A_off = ffi.flatten_ragged_f32(A_t, 1)
    p_flat, _ = ffi.flatten_ragged_f32(p_t, 1)
    q = FpiObs.apply(A_flat, p_flat, torch.as_tensor(obs, device="cuda"), A_off, O, S, deps, n)
    (q * cuda(r)).sum().backward()

    def loss(A64, p64):
        qs = ofpi.run_fpi_batch(A64, obs, p64, deps, n)
        return float(sum((qs[f] * r[:, sum(S[:f]):sum(S[:f + 1])]).sum() for f in range(len(S))))

    A64 = [a.astype(np.float64) for a in A]
    p64 = [p.astype(np.float64) for p in prior]
    scale = max(max(float(g.grad.abs().max()) for g in A_t), max(float(g.grad.abs().max()) for g in p_t))
    for m in range(len(O)):
        for b in range(batch):
            o = obs[b, m]
            for idx in list(np.ndindex(A[m].shape[2:]))[:6]:
                key = (b, o) + idx
                Ap = [a.copy() for a in A64]; Ap[m][key] += H
                Am = [a.copy() for a in A64]; Am[m][key] -= H
                fd = (loss(Ap, p64) - loss(Am, p64)) / (2 * H)
                got = float(A_t[m].grad[key])
                assert abs(got - fd) <= REL * max(scale, 1.0), (m, key, got, fd)
            # an unobserved row has no gradient
            assert float(A_t[m].grad[b, (o + 1) % O[m]].abs().max()) == 0.0
    for f in range(len(S)):
        for b in range(batch):
            for s in range(S[f]):
                pp = [x.copy() for x in p64]; pp[f][b, s] += H
                pm = [x.copy() for x in p64]; pm[f][b, s] -= H
                fd = (loss(A64, pp) - loss(A64, pm)) / (2 * H)
                got = float(p_t[f].grad[b, s])
                assert abs(got - fd) <= REL * max(scale, 1.0), (f, b, s, got, fd)


@pytest.mark.parametrize("case", [
    dict(S=[3, 2], O=[3, 4], U=[2, 2], T=2, A_deps=[[0, 1], [1]], B_deps=[[0], [1]], C2d=False),
    dict(S=[3, 4, 2], O=[4, 3], U=[2, 3, 1], T=2, A_deps=[[0, 2], [1, 2, 0]], B_deps=[[0], [1, 0], [2]], C2d=True),
])
def test_efe_adjoint_matches_finite_differences(case):
    from pymdp_b200 import ffi
    from pymdp_b200.autograd import NegEfe
    S, O, U, T = case["S"], case["O"], case["U"], case["T"]
    A_deps, B_deps = case["A_deps"], case["B_deps"]
    rng = np.random.default_rng(9)
    batch = 2
    A = [_dir(rng, (batch, O[m]) + tuple(S[d] for d in A_deps[m])) for m in range(len(O))]
    B = [_dir(rng, (batch, S[f]) + tuple(S[d] for d in B_deps[f]) + (U[f],)) for f in range(len(S))]
    C = [rng.normal(size=(batch, T, o)).astype(np.float32) for o in O]
    qs = [_dir(rng, (batch, s)) for s in S]
    pol = oefe.construct_policies(S, U, T)
    P = pol.shape[0]
    w = rng.normal(size=(batch, P))
    lay = ffi.EfeLayout(S, O, U, T, A_deps, B_deps)
    ts = {k: [cuda(x).requires_grad_(True) for x in v] for k, v in dict(A=A, B=B, C=C, qs=qs).items()}
    flat = {k: ffi.flatten_ragged_f32(v, 1)[0] for k, v in ts.items()}
    G = NegEfe.apply(flat["qs"], flat["A"], flat["B"], flat["C"], torch.as_tensor(pol, device="cuda").int(), lay, 3)
    (G * cuda(w)).sum().backward()

    base = {k: [x.astype(np.float64) for x in v] for k, v in dict(A=A, B=B, C=C, qs=qs).items()}

    def loss(d):
        tot = 0.0
        for b in range(batch):
            g = oefe.neg_efe_all_policies(pol, [q[b] for q in d["qs"]], [a[b] for a in d["A"]],
                                          [x[b] for x in d["B"]], [c[b] for c in d["C"]], A_deps, B_deps)
            tot += float((g * w[b]).sum())
        return tot

    scale = max(float(x.grad.abs().max()) for v in ts.values() for x in v)
    for k, arrs in base.items():
        for i, arr in enumerate(arrs):
            for key in [tuple(rng.integers(0, n) for n in arr.shape) for _ in range(5)]:
                dp = {kk: [x.copy() for x in vv] for kk, vv in base.items()}
                dm = {kk: [x.copy() for x in vv] for kk, vv in base.items()}
                dp[k][i][key] += H
                dm[k][i][key] -= H
                fd = (loss(dp) - loss(dm)) / (2 * H)
                got = float(ts[k][i].grad[key])
                assert abs(got - fd) <= REL * max(scale, 1.0), (k, i, key, got, fd)
