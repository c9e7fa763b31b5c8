"""FP64 restatement of the closed-loop rollout — TEST INFRASTRUCTURE ONLY.

One agent at a time, the reference's ``rollout`` (``pymdp/envs/rollout.py:
468-700``) for ``inference_algo="fpi"``, no learning, deterministic action
selection, with the agent's own A / B / D as its environment:

* reset: ``state_f ~ D_f``, ``obs_m ~ A_m[:, state]`` (``envs/env.py:333-350``);
* per step: prior = D at the first step, else ``B_f[..., a_prev] . qs_prev``
  (``rollout.py:65-84``, ``agent.py:825-851``); ``qs`` by FPI
  (``algos.py:88-155``, ``oracle.fpi``); ``G`` by ``oracle.efe``
  (``control.py:604-690``); ``q_pi = softmax(gamma G + log E)`` with E
  uniform; action = first step of the first maximum of ``q_pi``
  (``control.py:115-150``); ``state' ~ B[:, state, a]``, ``obs' ~
  A[:, state']`` (``envs/env.py:352-400``).

The environment's draws use the same counter-based generator as the CUDA
kernel: u = top 24 bits of SplitMix64 chained over (seed, agent, step,
stream) divided by 2^24, then an inverse-CDF pick with sequential float32
sums. SplitMix64 is Steele, Lea and Flood's published generator; the
reference draws with JAX's PRNG instead, which is not reproducible here.
"""

from __future__ import annotations

import numpy as np

from .efe import construct_policies, neg_efe_all_policies
from .fpi import log_stable, run_factorized_fpi, softmax

MASK = (1 << 64) - 1


def sm64(z: int) -> int:
    z = (z + 0x9E3779B97F4A7C15) & MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def u01(seed: int, agent: int, hstep: int, stream: int) -> np.float32:
    h = sm64(seed & MASK)
    for x in (agent, hstep, stream):
        h = sm64(h ^ (x & 0xFFFFFFFF))
    return np.float32(h >> 40) * np.float32(1.0 / 16777216.0)


def categorical32(p, u) -> int:
    """First i with float32 cumsum[i] > u * total (sequential sums)."""
    p = np.asarray(p, np.float32)
    total = np.float32(0.0)
    for v in p:
        total = np.float32(total + v)
    thr = np.float32(np.float32(u) * total)
    c = np.float32(0.0)
    for i, v in enumerate(p):
        c = np.float32(c + v)
        if c > thr:
            return i
    return len(p) - 1


def _obs(spec, state, seed, agent, hstep):
    out = []
    for m, (a, deps) in enumerate(zip(spec.A, spec.A_dependencies)):
        col = a[(slice(None),) + tuple(int(state[d]) for d in deps)]
        out.append(categorical32(col, u01(seed, agent, hstep, 64 + m)))
    return out


def reset(spec, seed, agent):
    state = [categorical32(d, u01(seed, agent, 0, f)) for f, d in enumerate(spec.D)]
    return state, _obs(spec, state, seed, agent, 0)


def env_step(spec, seed, agent, t, state, action):
    nxt = [categorical32(b[:, int(state[f]), int(action[f])], u01(seed, agent, t + 1, 128 + f))
           for f, b in enumerate(spec.B)]
    return nxt, _obs(spec, nxt, seed, agent, t + 1)


def plan(spec, qs, flags=3):
    """``(G, q_pi, action)`` for posterior ``qs``."""
    pol = construct_policies(spec.S, spec.U, spec.policy_len)
    A = [np.asarray(a, np.float64) for a in spec.A]
    B = [np.asarray(b, np.float64) for b in spec.B]
    C = [np.asarray(c, np.float64) for c in spec.C]
    G = neg_efe_all_policies(pol, qs, A, B, C, spec.A_dependencies, [[f] for f in range(len(spec.S))],
                             use_utility=bool(flags & 1), use_states_info_gain=bool(flags & 2))
    P = pol.shape[0]
    q_pi = softmax(spec.gamma * G + log_stable(np.full(P, 1.0 / P)))
    return G, q_pi, [int(x) for x in pol[int(np.argmax(q_pi)), 0]]


def infer(spec, obs, prior, num_iter):
    A = [np.asarray(a, np.float64) for a in spec.A]
    o = [np.eye(a.shape[0])[int(x)] for a, x in zip(A, obs)]
    return run_factorized_fpi(A, o, [np.asarray(p, np.float64) for p in prior], spec.A_dependencies, num_iter)


def rollout_agent(spec, agent, steps, seed, num_iter=16, flags=3, actions=None):
    """Per-step ``obs``, ``state``, ``qs``, ``G``, ``q_pi``, ``action``. With
    ``actions`` (``(steps, F)``) the environment follows those actions
    instead of the oracle's own, so a recorded trajectory can be replayed."""
    state, obs = reset(spec, seed, agent)
    prior = [np.asarray(d, np.float64) for d in spec.D]
    rec = {k: [] for k in ("obs", "state", "qs", "G", "q_pi", "action")}
    for t in range(steps):
        qs = infer(spec, obs, prior, num_iter)
        G, q_pi, act = plan(spec, qs, flags)
        for k, v in (("obs", obs), ("state", state), ("qs", qs), ("G", G), ("q_pi", q_pi), ("action", act)):
            rec[k].append(v)
        a = act if actions is None else [int(x) for x in actions[t]]
        prior = [np.asarray(b, np.float64)[:, :, a[f]] @ qs[f] for f, b in enumerate(spec.B)]
        state, obs = env_step(spec, seed, agent, t, state, a)
    return rec
