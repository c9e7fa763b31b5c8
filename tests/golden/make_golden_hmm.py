"""Generate the exact-HMM golden fixtures ``tests/golden/hmm_*.npz``.

Run in a container that holds the reference checkout::

    python tests/golden/make_golden_hmm.py /root/reference

Outputs come from the reference's own ``pymdp/algos.py``
(``run_exact_single_factor_hmm_scan``, ``hmm_filter_scan_colstoch``) and
``pymdp/inference.py`` (``smoothing_exact``), executed in float64 on NumPy
through ``refshim.py`` (its ``lax.associative_scan`` is a left fold in time
order, the same result for the associative combine), one sequence per call as
the reference vmaps them. Inputs are seeded and rounded to float32 first.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def cols(rng, shape, alpha=1.0):
    g = np.maximum(rng.gamma(alpha, size=shape), 1e-30)
    return f32(g / g.sum(0, keepdims=True))


def rows(rng, shape, alpha=1.0):
    g = np.maximum(rng.gamma(alpha, size=shape), 1e-30)
    return f32(g / g.sum(-1, keepdims=True))


# name -> (K, O list, U (0 = time-varying), T, distr_obs, Bn)
SCAN_CASES = {
    "hmm_scan_actions": (5, [4, 3], 3, 7, False, 3),
    "hmm_scan_distr": (6, [5], 2, 5, True, 2),
    "hmm_scan_time_varying": (4, [3, 2], 0, 6, False, 2),
    "hmm_scan_T1": (5, [4], 2, 1, False, 2),
    "hmm_scan_wide": (40, [12, 7], 4, 9, False, 2),
}

# name -> (K, U, T, Bn, invalid (agent, t) list)
SMOOTH_CASES = {
    "hmm_smoothing_exact": (6, 3, 8, 3, [(1, 2), (2, 0)]),
}


def make_scan_case(ref, cfg, seed):
    K, O, U, T, distr, Bn = cfg
    rng = np.random.default_rng(seed)
    A = [np.stack([cols(rng, (o, K), 0.7) for _ in range(Bn)]) for o in O]
    prior = rows(rng, (Bn, K))
    if U == 0:
        B = np.stack([np.stack([cols(rng, (K, K), 0.5) for _ in range(T - 1)]) for _ in range(Bn)])
        actions = None
    else:
        B = np.stack([cols(rng, (K, K, U), 0.5) for _ in range(Bn)])
        actions = rng.integers(0, U, size=(Bn, max(T - 1, 0)))
        if T > 2:
            actions[0, 1] = -1  # jnp indexing: the last action's transition
    if distr:
        obs = [rows(rng, (Bn, T, o), 0.5) for o in O]
    else:
        obs = [rng.integers(0, o, size=(Bn, T)) for o in O]
    out = {"K": np.array(K), "O": np.array(O), "U": np.array(U), "T": np.array(T), "distr": np.array(int(distr)),
           "Bn": np.array(Bn), "prior": prior, "B": B}
    if actions is not None:
        out["actions"] = actions
    mll, sm, pred, cond, filt = [], [], [], [], []
    for b in range(Bn):
        res = ref.algos.run_exact_single_factor_hmm_scan(
            [o[b] for o in obs], [a[b] for a in A], [B[b]], [prior[b]],
            actions=None if (actions is None or T == 1) else actions[b], distr_obs=distr)
        mll.append(res[0])
        sm.append(res[1][0])
        pred.append(res[2][0])
        cond.append(res[3][0])
        if U == 0 or T == 1:
            B_seq = B[b] if T > 1 else np.eye(K)
        else:
            B_seq = np.stack([B[b][:, :, u] for u in actions[b]])
        ll = np.stack([ref.maths.compute_log_likelihood([o[b][t] for o in obs], [a[b] for a in A],
                                                        distr_obs=distr) for t in range(T)])
        filt.append(ref.algos.hmm_filter_scan_colstoch(prior[b], B_seq, ll)[1])
    for m in range(len(O)):
        out[f"A{m}"], out[f"obs{m}"] = A[m], obs[m]
    out.update(mll=np.array(mll), smoothed=np.stack(sm), predicted=np.stack(pred), cond=np.stack(cond),
               filtered=np.stack(filt))
    return out


def make_smooth_case(ref, cfg, seed):
    K, U, T, Bn, invalid = cfg
    rng = np.random.default_rng(seed)
    B = np.stack([cols(rng, (K, K, U), 0.5) for _ in range(Bn)])
    filtered = rows(rng, (Bn, T, K), 0.8)
    actions = rng.integers(0, U, size=(Bn, T - 1))
    for b, t in invalid:
        actions[b, t] = -1
    sm, joint = [], []
    for b in range(Bn):
        s, j = ref.inference.smoothing_exact([filtered[b]], [B[b]], actions[b])
        sm.append(s[0])
        joint.append(j[0])
    return {"K": np.array(K), "U": np.array(U), "T": np.array(T), "Bn": np.array(Bn), "B": B,
            "filtered": filtered, "actions": actions, "smoothed": np.stack(sm), "joint": np.stack(joint)}


def main(ref_root):
    sys.path.insert(0, HERE)
    import refshim

    ref = refshim.load_reference(ref_root, modules=("utils", "maths", "algos", "inference"))
    for i, (name, cfg) in enumerate(SCAN_CASES.items()):
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make_scan_case(ref, cfg, 300 + i))
        print("wrote", name)
    for i, (name, cfg) in enumerate(SMOOTH_CASES.items()):
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make_smooth_case(ref, cfg, 400 + i))
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
