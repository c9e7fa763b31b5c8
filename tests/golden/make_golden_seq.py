"""Generate the sequence-inference golden fixtures ``tests/golden/seq_*.npz``.

Run in a container that holds the reference checkout::

    python tests/golden/make_golden_seq.py /root/reference

Outputs come from the reference's own ``run_mmp`` / ``run_vmp``
(``pymdp/algos.py:312-571``) executed in float64 on NumPy through
``refshim.py``, one sequence per call. Transitions are given as the
action-conditioned sequence ``(T-1, S_f, S_dep...)``. Inputs are seeded and
rounded to float32 first.
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


# name -> (kind, S, O, A_deps, B_deps, T, num_iter, tau, distr_obs)
CASES = {
    "seq_mmp": ("mmp", [3, 2], [4, 3], [[0, 1], [1]], [[0], [1, 0]], 5, 8, 0.25, True),
    "seq_mmp_index": ("mmp", [4, 3, 2], [5, 2], [[0, 2], [1]], [[0], [1], [2, 0]], 4, 6, 0.5, False),
    "seq_vmp": ("vmp", [3, 2], [4, 3], [[0, 1], [1]], [[0], [1, 0]], 5, 8, 0.25, True),
    "seq_vmp_index": ("vmp", [4, 3, 2], [5, 2], [[0, 2], [1]], [[0], [1], [2, 0]], 4, 6, 0.5, False),
    # the benchmark's window: 8 steps, S = [16, 8], both modalities on both factors, factor-local transitions
    "seq_mmp_bench": ("mmp", [16, 8], [16, 8], [[0, 1], [0, 1]], [[0], [1]], 8, 16, 0.25, False),
    "seq_vmp_bench": ("vmp", [16, 8], [16, 8], [[0, 1], [0, 1]], [[0], [1]], 8, 16, 0.25, False),
    # a modality on three factors, and a single-step window (no transition at all)
    "seq_mmp_rank3": ("mmp", [3, 4, 2], [5, 3], [[2, 0, 1], [1]], [[0, 1], [1], [2]], 4, 6, 0.5, True),
    "seq_vmp_t1": ("vmp", [5, 3], [4, 6], [[0], [0, 1]], [[0], [1]], 1, 5, 1.0, False),
}


def make_case(ref, cfg, seed):
    kind, S, O, A_deps, B_deps, T, num_iter, tau, distr = cfg
    rng = np.random.default_rng(seed)
    A = [cols(rng, (O[m],) + tuple(S[d] for d in A_deps[m]), 0.7) for m in range(len(O))]
    B = [np.moveaxis(cols(rng, (S[f], T - 1) + tuple(S[d] for d in B_deps[f]), 0.5), 1, 0) for f in range(len(S))]
    prior = [cols(rng, (s,), 1.0) for s in S]
    if distr:
        obs = [np.moveaxis(cols(rng, (O[m], T), 0.5), 1, 0) for m in range(len(O))]
    else:
        obs = [rng.integers(0, O[m], size=T) for m in range(len(O))]
    fn = ref.algos.run_mmp if kind == "mmp" else ref.algos.run_vmp
    qs = fn(A, B, obs, prior, A_deps, B_deps, num_iter=num_iter, tau=tau, distr_obs=distr)
    out = {"kind": np.array(kind), "S": np.array(S), "O": np.array(O), "T": np.array(T),
           "num_iter": np.array(num_iter), "tau": np.array(tau), "distr": np.array(int(distr)),
           "A_deps_flat": np.array([d for dd in A_deps for d in dd]), "A_deps_len": np.array([len(d) for d in A_deps]),
           "B_deps_flat": np.array([d for dd in B_deps for d in dd]), "B_deps_len": np.array([len(d) for d in B_deps])}
    for m in range(len(O)):
        out[f"A{m}"], out[f"obs{m}"] = A[m], obs[m]
    for f in range(len(S)):
        out[f"B{f}"], out[f"prior{f}"], out[f"qs{f}"] = B[f], prior[f], np.asarray(qs[f])
    return out


def main(ref_root, names=None):
    """Write every case, or only ``names`` (each case keeps its seed, 500 + its position in CASES)."""
    sys.path.insert(0, HERE)
    import refshim

    ref = refshim.load_reference(ref_root, modules=("utils", "maths", "algos"))
    for i, (name, cfg) in enumerate(CASES.items()):
        if names and name not in names:
            continue
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make_case(ref, cfg, 500 + i))
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference", sys.argv[2:] or None)
