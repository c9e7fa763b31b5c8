"""Generate the Dirichlet-learning golden fixtures ``tests/golden/learn_*.npz``.

Run in a container that holds the reference checkout::

    python tests/golden/make_golden_learning.py /root/reference

The outputs come from the reference's own ``pymdp/learning.py``
(``update_obs_likelihood_dirichlet``, ``update_state_transition_dirichlet``,
with ``pymdp/maths.py``'s ``multidimensional_outer`` and
``dirichlet_expected_value``) executed in float64 on NumPy through
``refshim.py``, called once per agent as ``Agent.infer_parameters`` vmaps them
(``pymdp/agent.py:569-607``). The transition joints are built as
``Agent.infer_parameters`` builds them for the filtering algorithms
(``agent.py:539-543``: ``[q_f[1:], q_dep[:-1] ...]``, each multiplied by
``valid_transition_mask``, ``agent.py:480-483, :502-511``). Inputs are drawn
from seeded generators and rounded to float32 first, so the float32 CUDA path
sees bit-identical values.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def dirichlet_cols(rng, shape, alpha=1.0):
    g = np.maximum(rng.gamma(alpha, size=shape), 1e-30)
    return f32(g / g.sum(0, keepdims=True))


def categorical(rng, n, lead=()):
    g = np.maximum(rng.gamma(1.0, size=lead + (n,)), 1e-30)
    return f32(g / g.sum(-1, keepdims=True))


# name -> (S, O, A_deps, T, categorical_obs, pA_none, lr, Bn)
A_CASES = {
    "learn_A_full": ([5, 3], [4, 6, 2], [[0, 1], [0, 1], [0, 1]], 1, False, [1], [1.0, 0.5, 2.0], 3),
    "learn_A_window": ([4, 3, 2], [3, 5, 2, 4], [[0], [1, 2], [0, 2], [2, 1, 0]], 4, False, [], [0.7, 1.3], 2),
    "learn_A_cat": ([4, 3], [3, 5, 2], [[0], [1], [0, 1]], 3, True, [], [0.25, 1.0, 4.0], 3),
    # a window longer than four steps and columns taller than sixteen rows
    "learn_A_long": ([20, 3], [24, 5], [[0], [0, 1]], 6, False, [], [0.9, 2.0], 2),
}

# name -> (S, U, B_deps, T, factors_to_update, lr, Bn, invalid (agent, t) list)
B_CASES = {
    "learn_B_online": ([4, 3, 2], [3, 1, 2], [[0], [1, 0], [2]], 2, "all", [1.0, 0.5, 2.0], 3, [(1, 0)]),
    "learn_B_window": ([5, 2, 3], [2, 2, 3], [[0, 2], [1], [2, 1, 0]], 5, [0, 2], [0.8, 1.5], 2, [(0, 2)]),
    "learn_B_long": ([18, 3], [2, 3], [[0], [1, 0]], 7, "all", [1.1, 0.6], 2, [(1, 3)]),
}


def make_A_case(ref, cfg, seed):
    S, O, deps, T, cat, none, lr, Bn = cfg
    rng = np.random.default_rng(seed)
    F, M = len(S), len(O)
    A = [np.stack([dirichlet_cols(rng, (O[m],) + tuple(S[f] for f in deps[m])) for _ in range(Bn)])
         for m in range(M)]
    pA = [f32(rng.uniform(0.05, 3.0, size=A[m].shape)) for m in range(M)]
    qs = [np.stack([categorical(rng, S[f], (T,)) for _ in range(Bn)]) for f in range(F)]
    if cat:
        obs = [np.stack([categorical(rng, O[m], (T,)) for _ in range(Bn)]) for m in range(M)]
    else:
        obs = [rng.integers(0, O[m], size=(Bn, T)).astype(np.int64) for m in range(M)]
        obs[0][0, 0] = -1  # out of range: one_hot gives zeros, nothing is added
    lr = f32(lr)
    qA_out = [np.zeros_like(a) for a in A]
    EA_out = [np.zeros_like(a) for a in A]
    for b in range(Bn):
        pA_b = [None if m in none else pA[m][b] for m in range(M)]
        o_b = [o[b] for o in obs]
        qA, EqA = ref.learning.update_obs_likelihood_dirichlet(
            pA_b, [a[b] for a in A], o_b, [q[b] for q in qs], A_dependencies=deps, categorical_obs=cat,
            num_obs=O, lr=lr[b])
        for m in range(M):
            qA_out[m][b] = pA[m][b] if qA[m] is None else qA[m]
            EA_out[m][b] = EqA[m]
    out = {"S": np.array(S), "O": np.array(O), "T": np.array(T), "categorical": np.array(int(cat)),
           "none_mask": np.array([int(m in none) for m in range(M)]), "lr": lr, "Bn": np.array(Bn),
           "deps_flat": np.array([d for dd in deps for d in dd]), "deps_len": np.array([len(d) for d in deps])}
    for m in range(M):
        out[f"A{m}"], out[f"pA{m}"], out[f"obs{m}"] = A[m], pA[m], obs[m]
        out[f"qA{m}"], out[f"EA{m}"] = qA_out[m], EA_out[m]
    for f in range(F):
        out[f"qs{f}"] = qs[f]
    return out


def make_B_case(ref, cfg, seed):
    S, U, deps, T, fts, lr, Bn, invalid = cfg
    rng = np.random.default_rng(seed)
    F = len(S)
    B = [np.stack([dirichlet_cols(rng, (S[f],) + tuple(S[d] for d in deps[f]) + (U[f],)) for _ in range(Bn)])
         for f in range(F)]
    pB = [f32(rng.uniform(0.05, 3.0, size=B[f].shape)) for f in range(F)]
    qs = [np.stack([categorical(rng, S[f], (T,)) for _ in range(Bn)]) for f in range(F)]
    actions = np.stack([rng.integers(0, U[f], size=(Bn, T - 1)) for f in range(F)], axis=-1).astype(np.int64)
    for b, t in invalid:
        actions[b, t, 0] = -1
    valid = np.all(actions >= 0, axis=-1).astype(np.float64)
    lr = f32(lr)
    qB_out = [np.zeros_like(x) for x in B]
    EB_out = [np.zeros_like(x) for x in B]
    for b in range(Bn):
        m = valid[b][:, None]
        joints = [[qs[f][b, 1:] * m] + [qs[d][b, :-1] * m for d in deps[f]] for f in range(F)]
        qB, EqB = ref.learning.update_state_transition_dirichlet(
            [p[b] for p in pB], [x[b] for x in B], joints, actions[b], num_controls=U, lr=lr[b],
            factors_to_update=fts)
        for f in range(F):
            qB_out[f][b], EB_out[f][b] = qB[f], EqB[f]
    fmask = (1 << F) - 1 if fts == "all" else sum(1 << f for f in fts)
    out = {"S": np.array(S), "U": np.array(U), "T": np.array(T), "factor_mask": np.array(fmask), "lr": lr,
           "Bn": np.array(Bn), "actions": actions, "deps_flat": np.array([d for dd in deps for d in dd]),
           "deps_len": np.array([len(d) for d in deps])}
    for f in range(F):
        out[f"B{f}"], out[f"pB{f}"], out[f"qs{f}"] = B[f], pB[f], qs[f]
        out[f"qB{f}"], out[f"EB{f}"] = qB_out[f], EB_out[f]
    return out


# name -> (S_f, S_prev, U, T, lr, Bn): learning from given pairwise joints, the
# smoothing algorithms' form (a joint array per factor, learning.py:153)
JOINT_CASES = {
    "learn_B_joint": (5, 5, 3, 6, [0.7, 1.4], 2),
}


def make_joint_case(ref, cfg, seed):
    S, Sp, U, T, lr, Bn = cfg
    rng = np.random.default_rng(seed)
    B = np.stack([dirichlet_cols(rng, (S, Sp, U)) for _ in range(Bn)])
    pB = f32(rng.uniform(0.05, 3.0, size=B.shape))
    g = np.maximum(rng.gamma(1.0, size=(Bn, T - 1, S, Sp)), 1e-30)
    joint = f32(g / g.sum(axis=(2, 3), keepdims=True))
    actions = rng.integers(0, U, size=(Bn, T - 1, 1)).astype(np.int64)
    actions[0, 1, 0] = -1  # one_hot gives zeros: this transition adds nothing
    lr = f32(lr)
    qB, EB = [], []
    for b in range(Bn):
        q, e = ref.learning.update_state_transition_dirichlet(
            [pB[b]], [B[b]], [joint[b]], actions[b], num_controls=[U], lr=lr[b])
        qB.append(q[0])
        EB.append(e[0])
    return {"U": np.array(U), "lr": lr, "Bn": np.array(Bn), "B": B, "pB": pB, "joint": joint, "actions": actions,
            "qB": np.stack(qB), "EB": np.stack(EB)}


def main(ref_root, names=None):
    sys.path.insert(0, HERE)
    import refshim

    ref = refshim.load_reference(ref_root, modules=("utils", "maths", "learning"))
    want = (lambda n: names is None or n in names)  # noqa: E731
    for i, (name, cfg) in enumerate(A_CASES.items()):
        if want(name):
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make_A_case(ref, cfg, 100 + i))
            print("wrote", name)
    for i, (name, cfg) in enumerate(B_CASES.items()):
        if want(name):
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make_B_case(ref, cfg, 200 + i))
            print("wrote", name)
    for i, (name, cfg) in enumerate(JOINT_CASES.items()):
        if want(name):
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make_joint_case(ref, cfg, 250 + i))
            print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference", sys.argv[2:] or None)
