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


def expected_state(qs, B, u_t, B_deps):
    """``control.py:351-389`` for all policies at once.

    ``qs[f]``: ``(P, S_f)``; ``u_t``: ``(P, F)`` actions; returns next ``qs``.
    """
    out = []
    for f, (B_f, deps) in enumerate(zip(B, B_deps)):
        # B_f[..., u] per policy: move the action axis first, gather.
        Bsel = np.moveaxis(np.asarray(B_f, np.float64), -1, 0)[u_t[:, f]]  # (P, S_f, *S_deps)
        r = len(deps)
        sub = _LET[: r + 1]
        subs = ["z" + sub] + ["z" + sub[j + 1] for j in range(r)]
        out.append(np.einsum(",".join(subs) + "->z" + sub[0], Bsel, *[qs[d] for d in deps], optimize=True))
    return out


def neg_efe_all_policies(policies, qs_init, A, B, C, A_deps, B_deps,
                         use_utility=True, use_states_info_gain=True):
    """``compute_neg_efe_policy`` (``control.py:604-690``) for every policy.

    Returns ``G`` of shape ``(P,)`` (``neg_efe``; larger is better).
    """
    policies = np.asarray(policies)
    P, T, F = policies.shape
    qs = [np.broadcast_to(np.asarray(q, np.float64), (P, len(q))) for q in qs_init]
    A = [np.asarray(a, np.float64) for a in A]
    H_A = [-stable_xlogx(a).sum(0) for a in A]
    G = np.zeros(P)
    for t in range(T):
        qs = expected_state(qs, B, policies[:, t, :], B_deps)
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
    return G


def update_posterior_policies(policies, qs_init, A, B, C, E, A_deps, B_deps, gamma=16.0,
                              use_utility=True, use_states_info_gain=True):
    """``control.py:198-349``: returns ``(q_pi, G)``."""
    G = neg_efe_all_policies(policies, qs_init, A, B, C, A_deps, B_deps,
                             use_utility=use_utility, use_states_info_gain=use_states_info_gain)
    return softmax(gamma * G + log_stable(E)), G


def sample_policy(policies, q_pi):
    """``control.py:115-150`` deterministic branch: first argmax, first step."""
    return np.asarray(policies)[int(np.argmax(q_pi)), 0]
