"""The agent loop's glue on the GPU: Agent.update_empirical_prior
(b2_expected_state; pymdp/agent.py:825-851 = control.compute_expected_state,
pymdp/control.py:351-389) and Agent.multiaction_probabilities
(b2_multiaction_probabilities; pymdp/agent.py:908-937) against the FP64
oracle. Tolerance: FP32 products, rtol 1e-5 / atol 1e-7 on probabilities."""

import numpy as np
import pytest
import torch

from oracle import efe as oefe

pytestmark = pytest.mark.gpu


def _model(rng, S, U, B_deps, batch):
    def dirc(shape, alpha=0.7):
        g = rng.gamma(alpha, size=shape) + 1e-30
        return (g / g.sum(1, keepdims=True)).astype(np.float32)
    B = [dirc((batch, S[f]) + tuple(S[d] for d in B_deps[f]) + (U[f],)) for f in range(len(S))]
    qs = [dirc((batch, s), 1.0) for s in S]
    return B, qs


@pytest.mark.parametrize("case", [
    dict(S=[4, 3, 5], U=[2, 3, 1], B_deps=[[0], [1], [2]]),
    dict(S=[3, 4, 2], U=[2, 3, 2], B_deps=[[0], [1, 0], [2, 1]]),
])
def test_update_empirical_prior_matches_oracle(case):
    from pymdp_b200 import Agent
    rng = np.random.default_rng(3)
    S, U, B_deps, batch = case["S"], case["U"], case["B_deps"], 6
    B, qs = _model(rng, S, U, B_deps, batch)
    A = [np.full((batch, 2) + tuple(S), 0.5, np.float32)]
    agent = Agent(A, B, B_dependencies=B_deps, batch_size=batch)
    act = np.stack([rng.integers(0, u, size=batch) for u in U], axis=1).astype(np.int32)
    act[0, 0] = -1          # negative: from the end, as jnp indexing
    act[1, 1] = U[1] + 3    # beyond U: clamped
    qs_d = [torch.as_tensor(q, device="cuda").unsqueeze(1) for q in qs]
    pred = agent.update_empirical_prior(torch.as_tensor(act, device="cuda"), qs_d)
    for b in range(batch):
        ref = oefe.expected_state([q[b:b + 1].astype(np.float64) for q in qs], [x[b] for x in B], act[b:b + 1],
                                  B_deps)
        for f in range(len(S)):
            np.testing.assert_allclose(pred[f][b].cpu().numpy(), ref[f][0], rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("mode", ["full", "marginal"])
@pytest.mark.parametrize("case", [
    dict(S=[3, 2, 2], U=[3, 2, 1], T=2),
    dict(S=[4, 3], U=[4, 3], T=1),
])
def test_multiaction_probabilities_matches_oracle(case, mode):
    from pymdp_b200 import Agent
    rng = np.random.default_rng(5)
    S, U, T, batch = case["S"], case["U"], case["T"], 4
    B, _ = _model(rng, S, U, [[f] for f in range(len(S))], batch)
    A = [np.full((batch, 2) + tuple(S), 0.5, np.float32)]
    agent = Agent(A, B, policy_len=T, batch_size=batch, sampling_mode=mode)
    pol = oefe.construct_policies(S, U, T)
    P = len(pol)
    g = rng.gamma(1.0, size=(batch, P))
    q_pi = (g / g.sum(1, keepdims=True)).astype(np.float32)
    out = agent.multiaction_probabilities(torch.as_tensor(q_pi, device="cuda")).cpu().numpy()
    assert out.shape == (batch, int(np.prod(U)))
    np.testing.assert_array_equal(agent.unique_multiactions.cpu().numpy(), oefe.unique_multiactions(pol, U))
    for b in range(batch):
        ref = oefe.multiaction_probabilities(q_pi[b], pol, U, mode)
        np.testing.assert_allclose(out[b], ref, rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(out[b].sum(), 1.0, rtol=1e-5)
