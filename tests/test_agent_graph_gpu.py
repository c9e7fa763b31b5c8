"""The agent step captured as CUDA graphs (``Agent.capture_step``) against
the same step called eagerly through ``Agent.infer_states`` ->
``infer_policies`` -> ``sample_action``: the graph replays the same kernels
on the same buffers, so qs, q_pi, G and the action are bitwise equal, over
several steps with new observations and priors each time, in the one-graph
and the two-graph (``split``) forms, on the factored and the dense paths.
The eager path itself is checked against the oracle in test_efe_gpu.py and
test_fpi_gpu.py."""

import numpy as np
import pytest
import torch

from pymdp_b200 import Agent

pytestmark = pytest.mark.gpu


def model(rng, S, O, U, batch):
    def cols(shape):
        g = rng.gamma(0.5, size=shape) + 1e-30
        return (g / g.sum(1, keepdims=True)).astype(np.float32)

    F = len(S)
    A = [cols((batch, o) + tuple(S)) for o in O]
    B = [cols((batch, s, s, u)) for s, u in zip(S, U)]
    C = [rng.normal(size=(batch, o)).astype(np.float32) for o in O]
    D = [np.full((batch, s), 1.0 / s, np.float32) for s in S]
    return A, B, C, D, F


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("algo,precision", [("factored", "fp32"), ("dense", "tf32x3")])
def test_graphed_step_equals_eager(split, algo, precision):
    rng = np.random.default_rng(7)
    S, O, U, batch = [6, 4, 3], [5, 7, 3], [3, 2, 1], 12
    A, B, C, D, F = model(rng, S, O, U, batch)
    agent = Agent(A, B, C=C, D=D, policy_len=2, gamma=16.0, batch_size=batch, num_iter=16, precision=precision,
                  efe_algorithm=algo)
    g = agent.capture_step(warmup=2, split=split)
    assert len(g.graphs) == (2 if split else 1)
    for step in range(3):
        obs = rng.integers(0, np.array(O), size=(batch, len(O))).astype(np.int32)
        prior = [rng.dirichlet(np.ones(s), size=batch).astype(np.float32) for s in S]
        qs_e = agent.infer_states(torch.as_tensor(obs, device="cuda"), [torch.as_tensor(p, device="cuda")
                                                                         for p in prior])
        q_pi_e, G_e = agent.infer_policies(qs_e)
        act_e = agent.sample_action(q_pi_e)
        # host inputs on even steps (copied in by step), device inputs on odd ones
        if step % 2 == 0:
            qs_g, q_pi_g, G_g, act_g = g.step(torch.as_tensor(obs).pin_memory(),
                                              [torch.as_tensor(p) for p in prior])
        else:
            qs_g, q_pi_g, G_g, act_g = g.step([torch.as_tensor(obs[:, m], device="cuda") for m in range(len(O))],
                                              torch.as_tensor(np.concatenate(prior, 1), device="cuda"))
        torch.cuda.synchronize()
        for f in range(F):
            assert torch.equal(qs_g[f], qs_e[f]), f"step {step} factor {f}"
        assert torch.equal(G_g, G_e), f"step {step}"
        assert torch.equal(q_pi_g, q_pi_e), f"step {step}"
        assert torch.equal(act_g, act_e), f"step {step}"


def test_graphed_step_rejects_stochastic_selection():
    rng = np.random.default_rng(1)
    A, B, C, D, _ = model(rng, [3, 2], [3, 2], [2, 1], 2)
    agent = Agent(A, B, C=C, D=D, batch_size=2, action_selection="stochastic")
    with pytest.raises(ValueError, match="deterministic"):
        agent.capture_step()


@pytest.mark.parametrize("algo,precision", [("factored", "fp32"), ("dense", "tf32x3")])
def test_pipelined_steps_equal_eager(algo, precision):
    """Agent.capture_pipeline alternates two buffer sets with the copies on
    side streams: every step's qs, q_pi, G and action (also the action copied
    into pinned host memory) equal the eager step on the same inputs,
    bitwise, while step k + 1's inputs are copied in during step k."""
    rng = np.random.default_rng(11)
    S, O, U, batch = [6, 4, 3], [5, 7, 3], [3, 2, 1], 12
    A, B, C, D, F = model(rng, S, O, U, batch)
    agent = Agent(A, B, C=C, D=D, policy_len=2, gamma=16.0, batch_size=batch, num_iter=16, precision=precision,
                  efe_algorithm=algo)
    pipe = agent.capture_pipeline(warmup=2)
    steps = 5
    obs = [rng.integers(0, np.array(O), size=(batch, len(O))).astype(np.int32) for _ in range(steps)]
    prior = [[rng.dirichlet(np.ones(s), size=batch).astype(np.float32) for s in S] for _ in range(steps)]
    want = []
    for k in range(steps):
        qs_e = agent.infer_states(torch.as_tensor(obs[k], device="cuda"),
                                  [torch.as_tensor(p, device="cuda") for p in prior[k]])
        q_pi_e, G_e = agent.infer_policies(qs_e)
        want.append(([q.clone() for q in qs_e], q_pi_e.clone(), G_e.clone(), agent.sample_action(q_pi_e).clone()))
    torch.cuda.synchronize()
    obs_h = [torch.as_tensor(o).pin_memory() for o in obs]
    prior_h = [torch.as_tensor(np.concatenate(p, 1)).pin_memory() for p in prior]
    act_h = [torch.empty((batch, F), dtype=torch.int32).pin_memory() for _ in range(steps)]
    got = []
    for k in range(steps):
        if k == 3:  # device inputs, made on the compute stream just before the step
            o_in, p_in = obs_h[k].cuda(), prior_h[k].cuda()
        else:
            o_in, p_in = obs_h[k], prior_h[k]
        qs_g, q_pi_g, G_g, act_g = pipe.step(o_in, p_in, act_h[k])
        # a step's outputs live until step k + 2 overwrites them: copy them out on the compute stream
        got.append(([q.clone() for q in qs_g], q_pi_g.clone(), G_g.clone(), act_g.clone()))
    pipe.drain()
    torch.cuda.synchronize()
    for k in range(steps):
        qs_e, q_pi_e, G_e, act_e = want[k]
        qs_g, q_pi_g, G_g, act_g = got[k]
        for f in range(F):
            assert torch.equal(qs_g[f], qs_e[f].reshape(qs_g[f].shape)), f"step {k} factor {f}"
        assert torch.equal(G_g, G_e), f"step {k}"
        assert torch.equal(q_pi_g, q_pi_e), f"step {k}"
        assert torch.equal(act_g, act_e), f"step {k}"
        assert torch.equal(act_h[k], act_e.cpu()), f"step {k}"
