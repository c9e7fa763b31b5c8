"""FP64 restatement of the reference's exact single-factor HMM inference — TEST INFRASTRUCTURE ONLY.

* ``log_likelihood``              ``pymdp/maths.py:214-263`` (``compute_log_likelihood``)
* ``select_transitions``          ``B0[:, :, u]`` of ``run_exact_single_factor_hmm_scan``
  (``pymdp/algos.py:1166-1196``, jnp indexing: a negative action counts from
  the end, then clamps) or ``invalid_action_mode="identity"`` of
  ``_condition_transitions_on_actions`` (``pymdp/inference.py:112-163``)
* ``hmm_filter``                  ``hmm_filter_scan_colstoch`` (``algos.py:959-988``,
  core ``:778-844``): the associative scan over conditioned transitions equals
  the time-ordered recursion p_0 = prior, p_t = B_{t-1} f_{t-1},
  f_t = p_t w_t / sum(p_t w_t) with w_t = exp(ll_t - max ll_t), and
  log p(o_{1:T}) = sum_t log sum(p_t w_t) + max ll_t (``_condition_on``,
  ``:750-775``)
* ``smoother_from_filtered``      ``hmm_smoother_from_filtered_colstoch`` (``:1049-1130``)
* ``run_exact_single_factor_hmm_scan``  ``:1132-1208``
* ``smoothing_exact``             ``pymdp/inference.py:595-634``

One sequence per call, float64 NumPy. Parity pin: checked against the golden
fixtures ``tests/golden/hmm_*.npz`` that ``tests/golden/make_golden_hmm.py``
produced by running the reference's own ``pymdp/algos.py`` and
``pymdp/inference.py``.
"""

from __future__ import annotations

import numpy as np

MINVAL = np.finfo(np.float64).eps


def log_stable(x):
    return np.log(np.maximum(x, MINVAL))


def log_likelihood(obs, A, distr_obs=True):
    """``(T, K)``: ``sum_m o_m[t] . log A_m`` or ``sum_m log A_m[o_m[t]]``;
    ``A[m]`` is ``(O_m, K)``; ``obs[m]`` is ``(T, O_m)`` or ``(T,)``."""
    T = np.shape(obs[0])[0]
    out = 0.0
    for o, a in zip(obs, A):
        la = log_stable(np.asarray(a, np.float64))
        if distr_obs:
            out = out + np.asarray(o, np.float64) @ la
        else:
            idx = np.asarray(o).astype(np.int64)
            idx = np.where(idx < 0, idx + a.shape[0], idx).clip(0, a.shape[0] - 1)
            out = out + la[idx]
    return np.broadcast_to(out, (T, np.shape(A[0])[1])).astype(np.float64)


def select_transitions(B0, actions, T, mode="index"):
    """``(T-1, K, K)`` transitions: ``B0`` 2-D (stationary), 3-D with an
    action axis (``actions`` given) or time-varying ``(T-1, K, K)``."""
    B0 = np.asarray(B0, np.float64)
    K = B0.shape[0] if B0.ndim != 3 or actions is not None else B0.shape[1]
    if B0.ndim == 2:
        return np.broadcast_to(B0, (max(T - 1, 0), K, K))
    if actions is None:
        return B0
    U = B0.shape[2]
    out = []
    for u in np.asarray(actions).reshape(-1).astype(np.int64):
        if mode == "identity" and u < 0:
            out.append(np.eye(K))
            continue
        if u < 0:
            u += U
        out.append(B0[:, :, int(np.clip(u, 0, U - 1))])
    return np.stack(out) if out else np.zeros((0, K, K))


def hmm_filter(prior, B_seq, ll):
    """Returns ``(mll, filtered (T, K), predicted (T, K))``."""
    T, K = ll.shape
    f = np.zeros((T, K))
    pred = np.zeros((T, K))
    mll = 0.0
    p = np.asarray(prior, np.float64)
    for t in range(T):
        if t > 0:
            p = B_seq[t - 1] @ f[t - 1]
        pred[t] = p
        m = ll[t].max()
        u = p * np.exp(ll[t] - m)
        c = u.sum()
        c = 1.0 if c == 0 else c
        f[t] = u / c
        mll += np.log(max(c, MINVAL)) + m
    return mll, f, pred


def smoother_from_filtered(filtered, B_seq):
    """Returns ``(smoothed (T, K), joint (T-1, K, K), cond (T-1, K, K))`` with
    ``joint[t, j, i] = p(s_{t+1}=j, s_t=i)``, ``cond[t, j, i] = p(s_t=i | s_{t+1}=j)``."""
    f = np.asarray(filtered, np.float64)
    T, K = f.shape
    if T == 1:
        return f.copy(), np.zeros((0, K, K)), np.zeros((0, K, K))
    pn = np.einsum("tji,ti->tj", B_seq, f[:-1])
    cond = B_seq * f[:-1][:, None, :] / np.maximum(pn[:, :, None], MINVAL)
    s = np.zeros((T, K))
    s[-1] = f[-1]
    for t in range(T - 2, -1, -1):
        s[t] = cond[t].T @ s[t + 1]
    sm = s / np.maximum(s.sum(-1, keepdims=True), MINVAL)
    joint = cond * sm[1:, :, None]
    return sm, joint, cond


def run_exact_single_factor_hmm_scan(obs, A, B, prior, actions=None, distr_obs=True):
    """``algos.py:1132-1208``: ``(mll, [smoothed], [predicted], [cond], filtered)``
    (the reference returns the first four)."""
    T = np.shape(obs[0])[0]
    B_seq = select_transitions(B[0], actions, T)
    ll = log_likelihood(obs, A, distr_obs)
    mll, f, pred = hmm_filter(prior[0], B_seq, ll)
    sm, _, cond = smoother_from_filtered(f, B_seq)
    return mll, [sm], [pred], [cond], f


def smoothing_exact(filtered_post, B, past_actions):
    """``inference.py:595-634``: ``([smoothed], [joint])`` with negative
    actions as identity transitions."""
    f = np.asarray(filtered_post[0], np.float64)
    B_seq = select_transitions(B[0], past_actions, f.shape[0], mode="identity")
    sm, joint, _ = smoother_from_filtered(f, B_seq)
    return [sm], [joint]
