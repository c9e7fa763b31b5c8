"""FP64 restatement of the reference's model-fitting action likelihood —
TEST INFRASTRUCTURE ONLY.

Per subject, ``evolve_trials`` (``pymdp/likelihoods.py:7-26``) scans over
trials:

* ``qs = agent.infer_states(o_t, prior)`` — FPI (``pymdp/algos.py:88-155``);
* ``q_pi = agent.infer_policies(qs)`` — ``softmax(gamma * G + log_stable(E))``
  (``pymdp/control.py:198-349``);
* ``probs = multiaction_probabilities(q_pi)`` (``pymdp/agent.py:908-937``,
  ``sampling_mode="full"``): the posterior mass of the policies whose first
  step is each unique multi-action. The unique multi-actions are the sorted
  unique rows of ``policies[:, 0]`` (``pymdp/agent.py:396-398``), which for a
  full policy set is the row-major order over ``num_controls``;
* ``prior = update_empirical_prior(a_t, qs)`` (``pymdp/agent.py:825-851``):
  ``B_f[..., a_t[f]] . qs`` for factor-local transitions
  (``pymdp/control.py:351-389``).

``aif_likelihood`` (``pymdp/likelihoods.py:28-45``) then scores the actions
with ``Categorical(logits=probs)``, i.e. it feeds the probabilities in as
logits. ``form="probs_as_logits"`` reproduces that; ``form="log"`` (default)
scores ``log probs[a_t]``, the action log-likelihood proper.

Model parameters are softmax logits for A (over the observation axis) and B
(over the next-state axis), raw C (log preferences) and ``log gamma``.

The FPI and EFE pieces are this package's ``fpi`` / ``efe`` functions, which
are pinned against the reference's own outputs; the composition has no
reference output to pin against here (the reference's likelihood needs JAX
and numpyro), so it follows the lines cited above.
"""

from __future__ import annotations

import numpy as np

from .efe import construct_policies, expected_state, neg_efe_all_policies
from .fpi import log_stable, run_factorized_fpi, softmax


def params_to_model(A_logits, B_logits):
    """Softmax of the logits: ``A[m]`` over axis 0, ``B[f]`` over axis 0."""
    A = [softmax(np.asarray(a, np.float64), axis=0) for a in A_logits]
    B = [softmax(np.asarray(b, np.float64), axis=0) for b in B_logits]
    return A, B


def multiaction_index(actions, num_controls):
    """Row-major index of each multi-action ``(…, F)`` over ``num_controls``."""
    idx = np.zeros(np.shape(actions)[:-1], dtype=np.int64)
    for f, u in enumerate(num_controls):
        idx = idx * int(u) + np.asarray(actions)[..., f]
    return idx


def multiaction_probabilities(q_pi, policies, num_controls):
    """``pymdp/agent.py:926-935`` (``sampling_mode="full"``)."""
    k = multiaction_index(np.asarray(policies)[:, 0, :], num_controls)
    out = np.zeros(int(np.prod(num_controls)))
    np.add.at(out, k, q_pi)
    return out


def subject_log_likelihood(A_logits, B_logits, C, log_gamma, obs, actions, num_controls, policy_len,
                           A_deps, num_iter, D=None, E=None, form="log"):
    """Summed action log-likelihood of one subject's trajectory.

    ``A_logits[m]``: ``(O_m, *S_deps)``; ``B_logits[f]``: ``(S_f, S_f, U_f)``
    (factor-local); ``C[m]``: ``(O_m,)``; ``obs``: ``(T, M)``; ``actions``:
    ``(T, F)``. ``D``/``E`` default to uniform.
    """
    A, B = params_to_model(A_logits, B_logits)
    S = [b.shape[0] for b in B]
    F = len(S)
    B_deps = [[f] for f in range(F)]
    policies = construct_policies(S, num_controls, policy_len)
    P = policies.shape[0]
    gamma = float(np.exp(log_gamma))
    prior = [np.full(s, 1.0 / s) for s in S] if D is None else [np.asarray(d, np.float64) for d in D]
    E = np.full(P, 1.0 / P) if E is None else np.asarray(E, np.float64)
    ll = 0.0
    for t in range(np.shape(obs)[0]):
        o = [np.eye(A[m].shape[0])[int(obs[t][m])] for m in range(len(A))]
        qs = run_factorized_fpi(A, o, prior, A_deps, num_iter)
        G = neg_efe_all_policies(policies, qs, A, B, [np.asarray(c, np.float64) for c in C], A_deps, B_deps)
        q_pi = softmax(gamma * G + log_stable(E))
        probs = multiaction_probabilities(q_pi, policies, num_controls)
        k = int(multiaction_index(np.asarray(actions[t]), num_controls))
        if form == "log":
            ll += float(np.log(probs[k]))
        elif form == "probs_as_logits":
            ll += float(probs[k] - np.log(np.exp(probs).sum()))
        else:
            raise ValueError(form)
        a = np.asarray(actions[t], np.int64)[None, :]
        prior = [p[0] for p in expected_state([q[None, :] for q in qs], B, a, B_deps)]
    return ll


def log_likelihood(A_logits, B_logits, C, log_gamma, obs, actions, num_controls, policy_len, A_deps, num_iter,
                   form="log"):
    """Sum over subjects; every argument carries a leading subject axis
    (``obs``: ``(N, T, M)``, ``actions``: ``(N, T, F)``)."""
    total = 0.0
    for n in range(np.shape(obs)[0]):
        total += subject_log_likelihood([a[n] for a in A_logits], [b[n] for b in B_logits], [c[n] for c in C],
                                        log_gamma[n], obs[n], actions[n], num_controls, policy_len, A_deps,
                                        num_iter, form=form)
    return total
