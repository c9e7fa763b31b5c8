"""FP64 restatement of the reference's online Dirichlet learning — TEST INFRASTRUCTURE ONLY.

* ``update_obs_likelihood_dirichlet``    ``pymdp/learning.py:11-117``
* ``update_state_transition_dirichlet``  ``pymdp/learning.py:119-233``
* ``dirichlet_expected_value``           ``pymdp/maths.py:843-862`` (clip at
  MINVAL, normalise over axis 0)
* ``update_state_transition_from_joint`` ``learning.py:119-157`` with given
  pairwise joints (the smoothing algorithms' form)
* ``infer_parameters``                   ``pymdp/agent.py:416-620`` for the
  filtering algorithms (``fpi`` / ``mmp`` / ``vmp``): A learns from the
  marginal beliefs, B from joints built out of the belief sequence
  (``agent.py:539-543``, ``:567``) masked by ``valid_transition_mask``
  (``agent.py:480-483``, ``:502-511``), and the B update is skipped for the
  whole batch unless some agent has a valid transition (``agent.py:486-500``).

One agent per call (the reference vmaps these over the batch); arrays are
float64 NumPy. Parity pin: checked against the golden fixtures that
``tests/golden/make_golden.py`` produced by running the reference's own
``pymdp/learning.py`` (``tests/golden/learn_*.npz``).
"""

from __future__ import annotations

from typing import Sequence

import numpy as np

MINVAL = np.finfo(np.float64).eps


def dirichlet_expected_value(p: np.ndarray) -> np.ndarray:
    """``maths.py:843-862``."""
    p = np.maximum(p, MINVAL)
    return p / p.sum(axis=0, keepdims=True)


def outer(vectors: Sequence[np.ndarray]) -> np.ndarray:
    """``maths.py:763-781`` (``multidimensional_outer``)."""
    x = np.asarray(vectors[0], dtype=np.float64)
    for v in vectors[1:]:
        x = x[..., None] * np.asarray(v, dtype=np.float64)
    return x


def one_hot(index, n: int) -> np.ndarray:
    """``jax.nn.one_hot``: all zeros for an index outside ``[0, n)``."""
    return (np.asarray(index)[..., None] == np.arange(n)).astype(np.float64)


def update_obs_likelihood_dirichlet(pA, A, obs, qs, A_dependencies, num_obs, lr=1.0, categorical_obs=False):
    """``learning.py:57-117`` for one agent. ``obs[m]``: ``(T,)`` indices or
    ``(T, O_m)`` distributions; ``qs[f]``: ``(T, S_f)``. ``pA[m]`` may be
    None (no update, ``A[m]`` kept). Returns ``(qA, E_qA)``."""
    qA, E_qA = [], []
    for m, pa in enumerate(pA):
        if pa is None:
            qA.append(None)
            E_qA.append(A[m])
            continue
        o = np.asarray(obs[m], dtype=np.float64) if categorical_obs else one_hot(obs[m], num_obs[m])
        T = o.shape[0]
        d = sum(outer([o[t]] + [qs[f][t] for f in A_dependencies[m]]) for t in range(T))
        new = np.asarray(pa, dtype=np.float64) + lr * d
        qA.append(new)
        E_qA.append(dirichlet_expected_value(new))
    return qA, E_qA


def update_state_transition_dirichlet(pB, B, joint_beliefs, actions, num_controls, lr=1.0,
                                      factors_to_update="all"):
    """``learning.py:159-233`` for one agent: ``joint_beliefs[f]`` is the list
    ``[q_f[1:], q_dep0[:-1], ...]`` (each ``(T-1, S)``), ``actions`` ``(T-1, F)``
    ints. Factors outside ``factors_to_update`` keep ``pB`` and get
    ``E[pB]``. Returns ``(qB, E_qB)``."""
    F = len(pB)
    chosen = range(F) if factors_to_update == "all" else sorted(factors_to_update)
    qB, E_qB = [], []
    for f in range(F):
        pb = np.asarray(pB[f], dtype=np.float64)
        if f in chosen:
            a = one_hot(np.asarray(actions)[:, f], num_controls[f])
            n = a.shape[0]
            d = sum(outer([j[t] for j in joint_beliefs[f]] + [a[t]]) for t in range(n))
            pb = pb + lr * d
        qB.append(pb)
        E_qB.append(dirichlet_expected_value(pb))
    return qB, E_qB


def update_state_transition_from_joint(pB_f, joint, actions_f, num_controls_f, lr=1.0):
    """``learning.py:119-157`` with a joint array (the smoothing algorithms'
    form, ``:153``): ``joint`` ``(T-1, S_f, S_prev...)`` pairwise posteriors,
    ``actions_f`` ``(T-1,)``; ``pB_f += lr * sum_t joint_t (x) onehot(a_t)``.
    Returns ``(qB_f, E_qB_f)``."""
    a = one_hot(np.asarray(actions_f), num_controls_f)
    d = sum(outer([np.asarray(joint[t], np.float64), a[t]]) for t in range(a.shape[0]))
    qb = np.asarray(pB_f, np.float64) + lr * d
    return qb, dirichlet_expected_value(qb)


def infer_parameters(pA, A, pB, B, beliefs_A, observations, actions, A_dependencies, B_dependencies, num_obs,
                     num_controls, learn_A=True, learn_B=True, beliefs_B=None, lr_pA=1.0, lr_pB=1.0,
                     categorical_obs=False):
    """``agent.py:416-620`` (filtering branch) for a BATCH: every array has a
    leading batch axis (``beliefs[f]``: ``(Bn, T, S_f)``, ``observations[m]``:
    ``(Bn, T)`` or ``(Bn, T, O_m)``, ``actions``: ``(Bn, F)`` or
    ``(Bn, T', F)``); ``lr_pA`` / ``lr_pB`` scalars or ``(Bn,)``. Returns
    ``(pA, A, pB, B)`` as lists of batched arrays (None where not learned)."""
    seq = beliefs_A if beliefs_B is None else beliefs_B
    Bn, T = seq[0].shape[0], seq[0].shape[1]
    if actions is not None:
        actions = np.asarray(actions)
        if actions.ndim == 2:
            actions = actions[:, None, :]
        actions = actions[:, :max(T - 1, 0), :]
        valid = np.all(actions >= 0, axis=-1)
    lrA = np.broadcast_to(np.asarray(lr_pA, dtype=np.float64), (Bn,))
    lrB = np.broadcast_to(np.asarray(lr_pB, dtype=np.float64), (Bn,))
    outA, outEA, outB, outEB = pA, A, pB, B
    if learn_A:
        per = [update_obs_likelihood_dirichlet(
            [None if p is None else p[b] for p in pA], [a[b] for a in A], [o[b] for o in observations],
            [q[b] for q in beliefs_A], A_dependencies, num_obs, lr=lrA[b], categorical_obs=categorical_obs)
            for b in range(Bn)]
        outA = [None if pA[m] is None else np.stack([per[b][0][m] for b in range(Bn)]) for m in range(len(pA))]
        outEA = [np.stack([per[b][1][m] for b in range(Bn)]) for m in range(len(A))]
    can_update_B = (learn_B and actions is not None and T > 1 and actions.shape[1] == T - 1
                    and bool(np.any(valid)))
    if can_update_B:
        per = []
        for b in range(Bn):
            m = valid[b].astype(np.float64)[:, None]
            joints = [[seq[f][b, 1:] * m] + [seq[d][b, :-1] * m for d in B_dependencies[f]]
                      for f in range(len(pB))]
            per.append(update_state_transition_dirichlet([p[b] for p in pB], [x[b] for x in B], joints, actions[b],
                                                         num_controls, lr=lrB[b]))
        outB = [np.stack([per[b][0][f] for b in range(Bn)]) for f in range(len(pB))]
        outEB = [np.stack([per[b][1][f] for b in range(Bn)]) for f in range(len(pB))]
    return outA, outEA, outB, outEB
