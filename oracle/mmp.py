"""FP64 restatement of the reference's sequence inference (MMP / VMP) — TEST INFRASTRUCTURE ONLY.

* ``run_mmp`` / ``run_vmp``   ``pymdp/algos.py:392-430, :512-571``, both through
  ``update_marginals`` (``:170-238``): log-marginals start at zero (uniform
  q), then ``num_iter`` mirror-descent steps
  ``ln q += tau * (ln A_marg - ln q + ln B_past + ln B_future)``,
  ``q = softmax(ln q - mean(ln q))`` (``mirror_gradient_descent_step``, ``:157-168``).
* ``ln A_marg``               ``all_marginal_log_likelihood`` (``:30-51``): per
  modality, its log-likelihood tensor contracted with every other dependency's
  marginal, summed over the modalities that depend on the factor.
* MMP messages                ``get_mmp_messages`` (``:432-510``): forward
  ``log E_q[B_t]`` (the prior at t = 0), backward ``log(q_{t+1} . B_norm)`` of
  the transition normalised over the current-state axis, each half-weighted
  on valid transitions.
* VMP messages                ``get_vmp_messages`` (``:312-390``): forward
  ``E_q[log B_t]`` (the prior at t = 0), backward ``q_{t+1} . E_q[log B_t]``.

Transitions are the action-conditioned sequence ``B[f]`` of shape
``(T-1, S_f, S_dep...)`` that ``_condition_transitions_on_actions`` produces.
No validity masks (a full window). One sequence per call, float64 NumPy.
Parity pin: ``tests/golden/seq_*.npz`` made by ``tests/golden/make_golden_seq.py``
from the reference's own ``pymdp/algos.py``.
"""

from __future__ import annotations

import numpy as np

MINVAL = np.finfo(np.float64).eps


def log_stable(x):
    return np.log(np.maximum(x, MINVAL))


def _softmax(x):
    e = np.exp(x - x.max(-1, keepdims=True))
    return e / e.sum(-1, keepdims=True)


def _contract_time(M, xs, axes, keep):
    """sum over every axis of M not in ``keep``; xs[i] ``(T', n)`` multiplies
    along (axis 0, axes[i]), sharing the leading time axis."""
    args = [M, list(range(M.ndim))]
    for x, a in zip(xs, axes):
        args += [x, [0, a]]
    return np.einsum(*args, list(keep))


def _log_likelihoods(obs_t, A, distr_obs):
    out = []
    for o, a in zip(obs_t, A):
        la = log_stable(np.asarray(a, np.float64))
        out.append(np.tensordot(np.asarray(o, np.float64), la, axes=(0, 0)) if distr_obs else la[int(o)])
    return out


def _marginal_ll(qs_t, lls_t, A_deps, S):
    """``all_marginal_log_likelihood`` at one time step."""
    out = [np.zeros(1) for _ in S]
    for ll, deps in zip(lls_t, A_deps):
        for l, f in enumerate(deps):
            args = [ll, list(range(ll.ndim))]
            for k, d in enumerate(deps):
                if k != l:
                    args += [qs_t[d], [k]]
            out[f] = out[f] + np.einsum(*args, [l])
    return out


def _messages(kind, B, qs, ln_prior, B_deps):
    """(ln_B_future, ln_B_past) per factor, each ``(T, S_f)``."""
    F = len(qs)
    T = qs[0].shape[0]
    fut, past = [], []
    for f in range(F):
        xs = [qs[d][:-1] for d in B_deps[f]]
        axes = [2 + i for i in range(len(B_deps[f]))]
        if kind == "mmp":
            msg = log_stable(_contract_time(B[f], xs, axes, (0, 1)))
        else:
            msg = _contract_time(log_stable(B[f]), xs, axes, (0, 1))
        msg = np.concatenate([ln_prior[f][None], msg], axis=0)
        if kind == "mmp":  # half of each valid edge here, half in the backward message
            msg = msg * np.where(np.arange(T) < T - 1, 0.5, 1.0)[:, None]
        fut.append(msg)
    for f in range(F):
        acc = np.zeros((max(T - 1, 0), qs[f].shape[1]))
        for i, deps in enumerate(B_deps):
            if f not in deps:
                continue
            pos = deps.index(f)
            others = [(d, 2 + j) for j, d in enumerate(deps) if d != f]
            M = B[i] if kind == "mmp" else log_stable(B[i])
            bm = _contract_time(M, [qs[d][:-1] for d, _ in others], [a for _, a in others], (0, 1, 2 + pos))
            q_next = qs[i][1:]
            if kind == "mmp":
                bn = bm / np.maximum(bm.sum(-1, keepdims=True), MINVAL)
                acc = acc + 0.5 * log_stable(np.einsum("ti,tif->tf", q_next, bn))
            else:
                acc = acc + np.einsum("ti,tif->tf", q_next, bm)
        past.append(np.concatenate([acc, np.zeros((1, qs[f].shape[1]))], axis=0))
    return fut, past


def run_sequence(kind, A, B, obs, prior, A_deps, B_deps, num_iter=1, tau=1.0, distr_obs=True):
    """``run_mmp`` (kind "mmp") or ``run_vmp`` (kind "vmp"): ``qs[f]`` ``(T, S_f)``."""
    S = [len(p) for p in prior]
    T = np.shape(obs[0])[0]
    lls = [_log_likelihoods([o[t] for o in obs], A, distr_obs) for t in range(T)]
    ln_prior = [log_stable(np.asarray(p, np.float64)) for p in prior]
    qs = [np.full((T, s), 1.0 / s) for s in S]
    B = [np.asarray(b, np.float64) for b in B]
    for _ in range(num_iter):
        ln_qs = [log_stable(q) for q in qs]
        fut, past = _messages(kind, B, qs, ln_prior, B_deps)
        ln_A = [[_marginal_ll([q[t] for q in qs], lls[t], A_deps, S)[f] for t in range(T)] for f in range(len(S))]
        new = []
        for f in range(len(S)):
            la = np.stack([np.broadcast_to(x, (S[f],)) for x in ln_A[f]])
            u = ln_qs[f] + tau * (la - ln_qs[f] + past[f] + fut[f])
            new.append(_softmax(u - u.mean(-1, keepdims=True)))
        qs = new
    return qs
