"""FP64 restatement of the reference's expected-free-energy policy evaluation.

Follows the pure-JAX branch of ``pymdp/control.py``:

* ``construct_policies``        ``control.py:152-195`` (itertools.product order)
* ``compute_expected_state``    ``control.py:351-389``
* ``compute_expected_obs``      ``control.py:420-447``
* ``compute_info_gain``         ``control.py:449-481`` (``H(qo) - sum_k H_A[k] x[k]``)
* ``compute_expected_utility``  ``control.py:483-509`` (C used raw; ``C[t]`` if 2-D)
* ``compute_neg_efe_policy``    ``control.py:604-690`` (scan over t from G=0)
* ``update_posterior_policies`` ``control.py:198-349``
  (``q_pi = softmax(gamma * G + log_stable(E))``)
* ``sample_policy``             ``control.py:115-150`` (deterministic: argmax,
  first maximum)
* parameter information gain  ``control.py:511-602`` (``calc_negative_pA_info_gain``,
  ``calc_negative_pB_info_gain``) with the exact Dirichlet weight
  ``spm_wnorm`` / ``_exact_wnorm`` (``maths.py:783-841``)
* inductive value             ``control.py:1021-1061`` (``calc_inductive_value_t``,
  anchored to ``qs_init``, ``control.py:775-777``) inside
  ``compute_neg_efe_policy_inductive`` (``control.py:692-793``)

with ``stable_xlogx(x) = xlogy(x, clip(x, MINVAL))`` (``maths.py:17-45``).
All policies are evaluated at once (vectorised over the policy axis); the
arithmetic per policy is the reference's.

Test infrastructure only (see ``oracle/__init__.py``).
"""

from __future__ import annotations

import itertools

import numpy as np

from .fpi import MINVAL, log_stable, softmax


def construct_policies(num_states, num_controls=None, policy_len=1, control_fac_idx=None):
    """``control.py:152-195``: ``(P, policy_len, F)`` int array."""
    F = len(num_states)
    if control_fac_idx is None:
        if num_controls is not None:
            control_fac_idx = [f for f, n in enumerate(num_controls) if n > 1]
        else:
            control_fac_idx = list(range(F))
    if num_controls is None:
        num_controls = [num_states[c] if c in control_fac_idx else 1 for c in range(F)]
    x = list(num_controls) * policy_len
    pols = list(itertools.product(*[range(i) for i in x]))
    return np.array(pols, dtype=np.int32).reshape(len(pols), policy_len, F)


def stable_xlogx(x):
    """``maths.py:17-30``."""
    x = np.asarray(x, np.float64)
    return x * np.log(np.clip(x, MINVAL, None))


_LET = "abcdefghijklmnopqrstuvwxyz"


def _joint(qs, deps):
    """Outer product of the dependency marginals per policy: ``(P, prod S)``,
    row-major over ``deps`` (the flattening of ``A_m``'s state axes)."""
    x = qs[deps[0]]
    for d in deps[1:]:
        x = (x[:, :, None] * qs[d][:, None, :]).reshape(x.shape[0], -1)
    return np.ascontiguousarray(x)


def jnp_index(u, n):
    """The element ``x[u]`` reads under JAX on an axis of size ``n``: a negative
    index counts from the end, then an out-of-bounds index is clamped (JAX's
    gather semantics; NumPy would raise)."""
    u = np.asarray(u)
    u = np.where(u < 0, u + n, u)
    return np.clip(u, 0, n - 1)


def expected_state(qs, B, u_t, B_deps):
    """``control.py:351-389`` for all policies at once.

    ``qs[f]``: ``(P, S_f)``; ``u_t``: ``(P, F)`` actions; returns next ``qs``.
    """
    out = []
    for f, (B_f, deps) in enumerate(zip(B, B_deps)):
        # B_f[..., u] per policy: move the action axis first, gather. The index
        # is read as a JAX gather reads it: negative from the end, then clamped.
        Bsel = np.moveaxis(np.asarray(B_f, np.float64), -1, 0)[jnp_index(u_t[:, f], B_f.shape[-1])]
        r = len(deps)
        sub = _LET[: r + 1]
        subs = ["z" + sub] + ["z" + sub[j + 1] for j in range(r)]
        out.append(np.einsum(",".join(subs) + "->z" + sub[0], Bsel, *[qs[d] for d in deps], optimize=True))
    return out


def exact_wnorm(a):
    """``maths.py:783-808`` (``_exact_wnorm``, the default of ``spm_wnorm``):
    ``-(log S - log a + 1/a - 1/S + digamma(a) - digamma(S))`` with ``a``
    clipped at MINVAL and ``S`` its clipped sum over axis 0."""
    from scipy.special import digamma

    a = np.clip(np.asarray(a, np.float64), MINVAL, None)
    s = np.clip(a.sum(axis=0), MINVAL, None)
    w = np.log(s) - np.log(a) + 1.0 / a - 1.0 / s + digamma(a) - digamma(s)
    return -w


def inductive_weights(qs_init, I, epsilon):
    """``calc_inductive_value_t`` (``control.py:1021-1061``) is linear in the
    predicted marginals: per factor ``path_available * (1 - I[m, :]) * log_eps``
    with ``idx = argmax qs_init[f]`` and ``m = max(argmax I[:, idx] - 1, 0)``
    (first maxima). Returns the weight vector of each factor."""
    log_eps = float(log_stable(np.float64(epsilon)))
    out = []
    for q, I_f in zip(qs_init, I):
        I_f = np.asarray(I_f, np.float64)
        idx = int(np.argmax(np.asarray(q)))
        m = max(int(np.argmax(I_f[:, idx])) - 1, 0)
        path = float(np.clip(I_f[:, idx].sum(0), 0, 1))
        out.append(path * (1.0 - I_f[m, :]) * log_eps)
    return out


def neg_efe_all_policies(policies, qs_init, A, B, C, A_deps, B_deps,
                         use_utility=True, use_states_info_gain=True, pA=None, pB=None,
                         use_param_info_gain=False, I=None, use_inductive=False, inductive_epsilon=1e-3):
    """``compute_neg_efe_policy`` (``control.py:604-690``) / its inductive
    variant (``control.py:692-793``) for every policy.

    Returns ``G`` of shape ``(P,)`` (``neg_efe``; larger is better). Per step:
    ``G += info_gain + utility - neg_param_info_gain + inductive_value``.
    """
    policies = np.asarray(policies)
    P, T, F = policies.shape
    qs = [np.broadcast_to(np.asarray(q, np.float64), (P, len(q))) for q in qs_init]
    A = [np.asarray(a, np.float64) for a in A]
    H_A = [-stable_xlogx(a).sum(0) for a in A]
    wA = ([exact_wnorm(pa) * (np.asarray(pa) > 0) for pa in pA]
          if (use_param_info_gain and pA is not None) else None)
    # pB weights per action slice: spm_wnorm(pB[..., u]) * (pB[..., u] > 0), stacked back on the last axis
    wB = None
    if use_param_info_gain and pB is not None:
        wB = []
        for pb in pB:
            pb = np.asarray(pb, np.float64)
            wB.append(np.stack([exact_wnorm(pb[..., u]) * (pb[..., u] > 0) for u in range(pb.shape[-1])], -1))
    wI = inductive_weights(qs_init, I, inductive_epsilon) if use_inductive else None
    G = np.zeros(P)
    for t in range(T):
        qs_prev = qs
        qs = expected_state(qs, B, policies[:, t, :], B_deps)
        if wB is not None:
            fd = expected_state(qs_prev, wB, policies[:, t, :], B_deps)  # factor_dot(wB[..., u], qs_prev)
            for f in range(F):
                G -= (qs[f] * fd[f]).sum(-1)
        if wI is not None:
            for f in range(F):
                G += qs[f] @ wI[f]
        joint = {}  # dependency tuple -> (P, K) matrix of x = outer product of the marginals
        for m, (A_m, deps) in enumerate(zip(A, A_deps)):
            key = tuple(deps)
            if key not in joint:
                joint[key] = _joint(qs, deps)
            x = joint[key]
            # factor_dot(A_m, qs[deps], keep_dims=(0,)) == A_m (O, K) . x (K,) per policy
            qo = x @ A_m.reshape(A_m.shape[0], -1).T                  # (P, O_m)
            if use_states_info_gain:
                H_qo = -stable_xlogx(qo).sum(-1)
                G += H_qo - x @ H_A[m].reshape(-1)
            if use_utility:
                C_m = np.asarray(C[m], np.float64)
                c = C_m[t] if C_m.ndim > 1 else C_m
                G += qo @ c
            if wA is not None:
                fd = x @ wA[m].reshape(wA[m].shape[0], -1).T           # factor_dot(wA_m, qs[deps])
                G -= (qo * fd).sum(-1)
    return G


def update_posterior_policies(policies, qs_init, A, B, C, E, A_deps, B_deps, gamma=16.0,
                              use_utility=True, use_states_info_gain=True, pA=None, pB=None,
                              use_param_info_gain=False, I=None, use_inductive=False, inductive_epsilon=1e-3):
    """``control.py:198-349`` / ``:795-963``: returns ``(q_pi, G)``."""
    G = neg_efe_all_policies(policies, qs_init, A, B, C, A_deps, B_deps,
                             use_utility=use_utility, use_states_info_gain=use_states_info_gain, pA=pA, pB=pB,
                             use_param_info_gain=use_param_info_gain, I=I, use_inductive=use_inductive,
                             inductive_epsilon=inductive_epsilon)
    return softmax(gamma * G + log_stable(E)), G


def sample_policy(policies, q_pi):
    """``control.py:115-150`` deterministic branch: first argmax, first step."""
    return np.asarray(policies)[int(np.argmax(q_pi)), 0]


def get_marginals(q_pi, policies, num_controls):
    """``control.py:42-67``: first-step action marginals, one per factor."""
    policies = np.asarray(policies)
    q_pi = np.asarray(q_pi, np.float64)
    return [np.array([q_pi[policies[:, 0, f] == a].sum() for a in range(int(u))])
            for f, u in enumerate(num_controls)]


def sample_action_marginal(policies, num_controls, q_pi):
    """Deterministic ``sample_action`` (``control.py:69-113``): first maximum
    of each factor's marginal."""
    return np.array([int(np.argmax(m)) for m in get_marginals(q_pi, policies, num_controls)])


def gumbel(seed, agent, factor, index):
    """Gumbel(0, 1) noise of the CUDA kernel's counter-based generator:
    u = (top 24 bits of SplitMix64 over (seed, agent, factor, index) + 0.5)
    / 2^24, g = -log(-log u)."""
    from .rollout import MASK, sm64
    h = sm64(seed & MASK)
    h = sm64(h ^ (agent & MASK))
    for x in (factor, index):
        h = sm64(h ^ (x & 0xFFFFFFFF))
    u = (np.float32(h >> 40) + np.float32(0.5)) * np.float32(1.0 / 16777216.0)
    return -np.log(-np.log(np.float64(u)))


def sample_stochastic(logits_base, alpha, seed, agent, factor):
    """Gumbel-max draw from the categorical with logits alpha * log clip(x)
    (the method of jax.random.categorical), with the kernel's noise. Returns
    (index, gap between the two largest perturbed logits)."""
    x = np.asarray(logits_base, np.float64)
    z = alpha * log_stable(x) + np.array([gumbel(seed, agent, factor, i) for i in range(len(x))])
    top = np.sort(z)
    gap = top[-1] - top[-2] if len(top) > 1 else np.inf
    return int(np.argmax(z)), gap


def unique_multiactions(policies, num_controls):
    """``Agent.unique_multiactions`` (``pymdp/agent.py:396-399``): sorted distinct
    rows of ``policies[:, 0]``, padded with -1 rows to ``prod(num_controls)``."""
    first = np.unique(np.asarray(policies)[:, 0], axis=0)
    size = int(np.prod(num_controls))
    out = np.full((size, first.shape[1]), -1, dtype=np.int64)
    out[:min(size, len(first))] = first[:size]
    return out


def multiaction_probabilities(q_pi, policies, num_controls, sampling_mode="full"):
    """``Agent.multiaction_probabilities`` (``pymdp/agent.py:908-937``) for one
    agent: "marginal" = the outer products of ``get_marginals``
    (``control.py:42-67``) reduced left to right; "full" = q_pi summed where
    ``policies[:, 0]`` equals each unique multi-action."""
    q_pi = np.asarray(q_pi, np.float64)
    if sampling_mode == "marginal":
        m = get_marginals(q_pi, policies, num_controls)
        out = m[0]
        for x in m[1:]:
            out = np.outer(out, x).reshape(-1)
        return out
    uniq = unique_multiactions(policies, num_controls)
    locs = np.all(np.asarray(policies)[:, 0] == uniq[:, None, :], axis=-1)  # (n_unique, P)
    return np.where(locs, q_pi[None, :], 0.0).sum(-1)
