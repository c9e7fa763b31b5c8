"""FP64 restatement of the reference's factorized fixed-point iteration.

Follows ``pymdp/algos.py:88-155`` (``run_factorized_fpi``) and the JAX body it
dispatches to the FFI with (``pymdp/algos.py:121-133``), plus the helpers in
``pymdp/maths.py``:

* ``MINVAL = finfo(float64).eps``                  (``maths.py:15``)
* ``log_stable(x) = log(clip(x, MINVAL))``         (``maths.py:64-79``)
* ``ll_m = tensordot(o_m, log_stable(A_m), [[0],[0]])`` (``maths.py:214-238``)
* per-factor marginal of each modality's log-likelihood against the other
  factors' marginals                                 (``algos.py:26-51``)
* Jacobi update ``log_q_f = log_prior_f + sum_m mll_{m,f}(q)`` from
  ``log_q = 0``, ``num_iter`` times, no early stop, final softmax
  (``algos.py:140-155``); single-factor models take the exact one-pass
  softmax (``algos.py:100-104``).

Test infrastructure only (see ``oracle/__init__.py``).
"""

from __future__ import annotations

import numpy as np

MINVAL = float(np.finfo(np.float64).eps)


def log_stable(x):
    """``maths.py:64-79``: ``log(clip(x, MINVAL))``."""
    return np.log(np.clip(np.asarray(x, dtype=np.float64), MINVAL, None))


def softmax(x, axis=-1):
    """``jax.nn.softmax``: ``exp(x - max) / sum``."""
    x = np.asarray(x, dtype=np.float64)
    e = np.exp(x - np.max(x, axis=axis, keepdims=True))
    return e / np.sum(e, axis=axis, keepdims=True)


def log_likelihood_single(o_m, A_m):
    """``maths.py:214-238`` with ``distr_obs=True``."""
    return np.tensordot(np.asarray(o_m, np.float64), log_stable(A_m), axes=([0], [0]))


def _marginal(ll_m, qs_deps, keep):
    """``algos.py:26-28``: contract ``ll_m`` with every dep marginal except ``keep``."""
    letters = "abcdefghij"[: ll_m.ndim]
    ops = [ll_m]
    subs = [letters]
    for j, q in enumerate(qs_deps):
        if j == keep:
            continue
        ops.append(q)
        subs.append(letters[j])
    return np.einsum(",".join(subs) + "->" + letters[keep], *ops)


def fpi_from_ll(ll, log_prior, A_deps, num_iter):
    """The JAX FPI body the reference hands to its FFI (``algos.py:121-133``).

    ``ll``: list of M arrays, ``ll[m]`` of shape ``S[A_deps[m]]``.
    ``log_prior``: list of F arrays of shape ``(S_f,)``.
    Returns the list of F posterior marginals.
    """
    F = len(log_prior)
    lp = [np.asarray(x, np.float64) for x in log_prior]
    ll = [np.asarray(x, np.float64) for x in ll]
    log_q = [np.zeros_like(x) for x in lp]
    for _ in range(num_iter):
        q = [softmax(x) for x in log_q]
        acc = [np.zeros_like(x) for x in lp]
        for m, deps in enumerate(A_deps):
            qd = [q[d] for d in deps]
            for i, f in enumerate(deps):
                acc[f] = acc[f] + _marginal(ll[m], qd, i)
        log_q = [acc[f] + lp[f] for f in range(F)]
    return [softmax(x) for x in log_q]


def run_factorized_fpi(A, obs, prior, A_deps, num_iter):
    """``algos.py:88-155`` for one agent (``obs`` are distributions)."""
    if len(prior) == 1:
        ll = sum(log_likelihood_single(o, a) for o, a in zip(obs, A))
        return [softmax(ll + log_stable(prior[0]))]
    ll = [log_likelihood_single(o, a) for o, a in zip(obs, A)]
    return fpi_from_ll(ll, [log_stable(p) for p in prior], A_deps, num_iter)


def one_hot(o, n):
    """``jax.nn.one_hot(o, n)`` as ``Agent.make_categorical`` uses it
    (``pymdp/agent.py:659-673``): all zeros for an index outside [0, n)."""
    return (np.arange(n) == int(o)).astype(np.float64)


def run_fpi_batch(A, obs_idx, prior, A_deps, num_iter):
    """Batched convenience wrapper (one-hot observations given as indices).

    ``A[m]``: ``(batch, O_m, *S_deps)`` or ``(O_m, *S_deps)`` (shared).
    ``obs_idx``: ``(batch, M)`` int. ``prior[f]``: ``(batch, S_f)``.
    Returns list of F arrays ``(batch, S_f)``.
    """
    batch = obs_idx.shape[0]
    F = len(prior)
    out = [np.zeros((batch, np.shape(prior[f])[-1])) for f in range(F)]
    for b in range(batch):
        A_b = [a[b] if a.ndim == len(A_deps[m]) + 2 else a for m, a in enumerate(A)]
        obs = [one_hot(obs_idx[b, m], A_b[m].shape[0]) for m in range(len(A))]
        pr = [p[b] for p in prior]
        qs = run_factorized_fpi(A_b, obs, pr, A_deps, num_iter)
        for f in range(F):
            out[f][b] = qs[f]
    return out
