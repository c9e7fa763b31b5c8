"""Generate the golden fixtures in ``tests/golden/*.npz`` from the reference.

Run in a container that holds the reference checkout::

    python tests/golden/make_golden.py /root/reference

Every fixture's outputs come from the reference's own code —
``pymdp/algos.py::run_factorized_fpi`` and
``pymdp/control.py::update_posterior_policies`` /
``construct_policies`` / ``sample_policy`` — executed in float64 on NumPy via
``refshim.py`` (JAX is not installed here). Inputs are drawn from seeded
``numpy.random.default_rng`` generators and rounded to float32 before the
reference sees them, so the float32 CUDA path and the FP64 reference consume
bit-identical values.

The cases follow the reference's own test shapes (``test/test_inference_jax.py``,
``test/test_control_jax.py``, ``perf_fixtures/fpi_large.py``) and the benchmark
configurations (plain single agent; rank-2 batched FPI; the EFE model with
S=[32,16,8], U=[4,4,1], O=[16,16,8,8,4]).
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def dirichlet_cols(rng, shape, alpha):
    """Columns (axis 0) ~ Dirichlet(alpha), float32-exact."""
    g = rng.gamma(alpha, size=shape)
    g = np.maximum(g, 1e-30)
    return f32(g / g.sum(0, keepdims=True))


def uniform_cols(rng, shape):
    u = rng.uniform(size=shape)
    return f32(u / u.sum(0, keepdims=True))


def pack(prefix, arrays):
    return {f"{prefix}{i}": np.asarray(a) for i, a in enumerate(arrays)}


def deps_arrays(deps):
    flat = np.array([d for ds in deps for d in ds], dtype=np.int64)
    offs = np.cumsum([0] + [len(ds) for ds in deps]).astype(np.int64)
    return flat, offs


# ---------------------------------------------------------------- FPI cases
FPI_CASES = {
    # plain single agent (benchmark config 1)
    "fpi_plain": dict(S=[3, 2], O=[3, 5], deps=[[0, 1], [0, 1]], batch=1, A="uniform",
                      prior="uniform", seed=1),
    # single factor: reference's exact one-pass branch (algos.py:100-104)
    "fpi_single_factor": dict(S=[7], O=[5, 3], deps=[[0], [0]], batch=3, A="dir1", prior="dir1", seed=2),
    # mixed ranks 1/2/3 (perf_fixtures/fpi_large.py layout, shrunk)
    "fpi_rank123": dict(S=[6, 5, 4], O=[4, 7, 3, 5], deps=[[0], [0, 1], [1, 2], [0, 1, 2]],
                        batch=4, A="dir05", prior="dir1", seed=3),
    # rank 4 and permuted dependency order
    "fpi_rank4": dict(S=[3, 4, 2, 5], O=[6, 4], deps=[[2, 0, 3, 1], [3, 1]], batch=3, A="dir05",
                      prior="dir1", seed=4),
    # factor without any modality keeps its prior
    "fpi_orphan_factor": dict(S=[4, 3, 5], O=[6], deps=[[2, 0]], batch=2, A="dir1", prior="dir1", seed=5),
    # benchmark config 2 shape (4 x 16 states, 6 x 32 obs, rank-2 deps), few agents
    "fpi_cfg2": dict(S=[16, 16, 16, 16], O=[32] * 6, deps="rank2_random", batch=2, A="dir05",
                     prior="dir1", seed=6),
    # perf_fixtures/fpi_large.py shapes
    "fpi_large": dict(S=[32, 24, 16], O=[16, 32, 8], deps=[[0, 1], [1, 2], [0, 1, 2]], batch=1,
                      A="dir1", prior="uniform", seed=7),
}


def make_fpi_case(ref, name, cfg):
    rng = np.random.default_rng(cfg["seed"])
    S, O = cfg["S"], cfg["O"]
    M, F = len(O), len(S)
    deps = cfg["deps"]
    if deps == "rank2_random":
        deps = [sorted(rng.choice(F, size=2, replace=False).tolist()) for _ in range(M)]
    batch = cfg["batch"]
    A = []
    for m in range(M):
        shape = (batch, O[m]) + tuple(S[d] for d in deps[m])
        if cfg["A"] == "uniform":
            a = np.stack([uniform_cols(rng, shape[1:]) for _ in range(batch)])
        else:
            alpha = {"dir05": 0.5, "dir1": 1.0}[cfg["A"]]
            a = np.stack([dirichlet_cols(rng, shape[1:], alpha) for _ in range(batch)])
        A.append(a)
    if cfg["prior"] == "uniform":
        prior = [f32(np.ones((batch, s)) / s) for s in S]
    else:
        prior = [np.stack([dirichlet_cols(rng, (s,), 1.0) for _ in range(batch)]) for s in S]
    obs = rng.integers(0, np.array(O), size=(batch, M)).astype(np.int32)
    num_iter = 16
    qs = [np.zeros((batch, s)) for s in S]
    ll = [np.zeros((batch,) + tuple(S[d] for d in deps[m])) for m in range(M)]
    for b in range(batch):
        o_vec = [np.eye(O[m])[obs[b, m]] for m in range(M)]
        out = ref.algos.run_factorized_fpi([a[b] for a in A], o_vec, [p[b] for p in prior], deps,
                                           num_iter=num_iter)
        for f in range(F):
            qs[f][b] = out[f]
        for m in range(M):
            ll[m][b] = ref.maths.compute_log_likelihood_single_modality(o_vec[m], A[m][b])
    dep_flat, dep_offs = deps_arrays(deps)
    data = dict(S=np.array(S, np.int64), O=np.array(O, np.int64), A_dep_flat=dep_flat,
                A_dep_offsets=dep_offs, num_iter=np.int64(num_iter), obs=obs)
    data.update(pack("A", [a.astype(np.float32) for a in A]))
    data.update(pack("prior", [p.astype(np.float32) for p in prior]))
    data.update(pack("qs", qs))
    data.update(pack("ll", ll))
    return data


# ---------------------------------------------------------------- EFE cases
EFE_CASES = {
    # benchmark config 1: plain single agent, gamma 16, T=1
    "efe_plain": dict(S=[3, 2], O=[3, 5], U=[3, 1], T=1, A_deps=None, B_deps=None, A="uniform",
                      B="uniform", C="uniform", E="uniform", qs="uniform", seed=11),
    # mixed A deps, factor-local B, time-indexed C on one modality, random E
    "efe_mixed": dict(S=[4, 3, 2], O=[5, 3, 4], U=[3, 2, 1], T=2, A_deps=[[0], [0, 1], [1, 2]],
                      B_deps=None, A="dir05", B="dir05", C="normal_t", E="dir1", qs="dir1", seed=12),
    # multi-parent B dependencies
    "efe_bdeps": dict(S=[3, 4, 2], O=[4, 5], U=[2, 3, 2], T=2, A_deps=[[0, 2], [1, 2, 0]],
                      B_deps=[[0], [1, 0], [2, 1]], A="dir05", B="dir05", C="normal", E="uniform",
                      qs="dir1", seed=13),
    # benchmark config 3 model (S=[32,16,8], U=[4,4,1], O=[16,16,8,8,4]), horizon 1
    "efe_cfg3_t1": dict(S=[32, 16, 8], O=[16, 16, 8, 8, 4], U=[4, 4, 1], T=1, A_deps=None,
                        B_deps=None, A="dir05", B="dir05", C="normal", E="uniform", qs="dir1", seed=14),
    # same model family, smaller states, full horizon 3 (P = 4096)
    "efe_cfg3_small": dict(S=[8, 4, 2], O=[16, 16, 8, 8, 4], U=[4, 4, 1], T=3, A_deps=None,
                           B_deps=None, A="dir05", B="dir05", C="normal", E="uniform", qs="dir1",
                           seed=15),
}


def make_efe_case(ref, name, cfg):
    rng = np.random.default_rng(cfg["seed"])
    S, O, U, T = cfg["S"], cfg["O"], cfg["U"], cfg["T"]
    F, M = len(S), len(O)
    A_deps = cfg["A_deps"] or [list(range(F)) for _ in range(M)]
    B_deps = cfg["B_deps"] or [[f] for f in range(F)]
    A = []
    for m in range(M):
        shape = (O[m],) + tuple(S[d] for d in A_deps[m])
        A.append(uniform_cols(rng, shape) if cfg["A"] == "uniform" else dirichlet_cols(rng, shape, 0.5))
    B = []
    for f in range(F):
        shape = (S[f],) + tuple(S[d] for d in B_deps[f]) + (U[f],)
        B.append(uniform_cols(rng, shape) if cfg["B"] == "uniform" else dirichlet_cols(rng, shape, 0.5))
    C = []
    for m in range(M):
        if cfg["C"] == "uniform":
            C.append(f32(np.ones(O[m]) / O[m]))
        elif cfg["C"] == "normal_t" and m == 1:
            C.append(f32(rng.normal(size=(T, O[m]))))
        else:
            C.append(f32(rng.normal(size=O[m])))
    policies = np.asarray(ref.control.construct_policies(S, U, T)).astype(np.int32)
    P = policies.shape[0]
    E = f32(np.ones(P) / P) if cfg["E"] == "uniform" else dirichlet_cols(rng, (P,), 1.0)
    if cfg["qs"] == "uniform":
        qs = [f32(np.ones(s) / s) for s in S]
    else:
        qs = [dirichlet_cols(rng, (s,), 1.0) for s in S]
    gamma = 16.0
    q_pi, G = ref.control.update_posterior_policies(policies, qs, A, B, C, E, None, None, A_deps,
                                                    B_deps, gamma=gamma)
    action = np.asarray(ref.control.sample_policy(policies, q_pi))
    adf, ado = deps_arrays(A_deps)
    bdf, bdo = deps_arrays(B_deps)
    data = dict(S=np.array(S, np.int64), O=np.array(O, np.int64), U=np.array(U, np.int64),
                T=np.int64(T), A_dep_flat=adf, A_dep_offsets=ado, B_dep_flat=bdf, B_dep_offsets=bdo,
                policies=policies, E=E.astype(np.float32), gamma=np.float64(gamma),
                q_pi=np.asarray(q_pi, np.float64), G=np.asarray(G, np.float64),
                action=action.astype(np.int32), C_ndim=np.array([np.ndim(c) for c in C], np.int64))
    data.update(pack("A", [a.astype(np.float32) for a in A]))
    data.update(pack("B", [b.astype(np.float32) for b in B]))
    data.update(pack("C", [c.astype(np.float32) for c in C]))
    data.update(pack("qs", [q.astype(np.float32) for q in qs]))
    return data


# EFE with the flag-gated terms: parameter information gain (pA / pB) and the
# inductive value (I from the reference's own generate_I_matrix)
EFE_EXTRA_CASES = {
    "efe_pig": dict(S=[3, 4, 2], O=[4, 5, 3], U=[2, 3, 2], T=2, A_deps=[[0, 2], [1], [1, 2, 0]],
                    B_deps=[[0], [1, 0], [2]], pA=True, pB=True, ind=False, seed=21),
    "efe_pigA": dict(S=[4, 3], O=[6, 2], U=[3, 2], T=2, A_deps=[[0, 1], [1]], B_deps=[[0], [1]],
                     pA=True, pB=False, ind=False, seed=22),
    "efe_ind": dict(S=[5, 4, 3], O=[4, 3], U=[3, 2, 1], T=3, A_deps=[[0, 1], [2, 1]], B_deps=[[0], [1], [2]],
                    pA=False, pB=False, ind=True, seed=23),
    "efe_all": dict(S=[4, 3, 2], O=[3, 4], U=[2, 3, 2], T=2, A_deps=[[0, 1], [2, 0]], B_deps=[[0], [1], [2]],
                    pA=True, pB=True, ind=True, seed=24),
}


def dirichlet_counts(rng, shape):
    """Positive concentration-like counts with about a tenth set to zero (the
    (pA > 0) mask of the reference's weight)."""
    a = rng.gamma(2.0, size=shape) * 3.0
    a[rng.random(size=shape) < 0.1] = 0.0
    return f32(a)


def make_efe_extra_case(ref, name, cfg):
    rng = np.random.default_rng(cfg["seed"])
    S, O, U, T = cfg["S"], cfg["O"], cfg["U"], cfg["T"]
    F, M = len(S), len(O)
    A_deps, B_deps = cfg["A_deps"], cfg["B_deps"]
    A = [dirichlet_cols(rng, (O[m],) + tuple(S[d] for d in A_deps[m]), 0.5) for m in range(M)]
    B = [dirichlet_cols(rng, (S[f],) + tuple(S[d] for d in B_deps[f]) + (U[f],), 0.5) for f in range(F)]
    C = [f32(rng.normal(size=O[m])) for m in range(M)]
    qs = [dirichlet_cols(rng, (s,), 1.0) for s in S]
    policies = np.asarray(ref.control.construct_policies(S, U, T)).astype(np.int32)
    P = policies.shape[0]
    E = dirichlet_cols(rng, (P,), 1.0)
    pA = [dirichlet_counts(rng, a.shape) for a in A] if cfg["pA"] else None
    pB = [dirichlet_counts(rng, b.shape) for b in B] if cfg["pB"] else None
    use_pig = cfg["pA"] or cfg["pB"]
    eps = 1e-3
    if cfg["ind"]:
        H = [f32(np.eye(s)[rng.integers(s)]) for s in S]
        I = [np.asarray(i, np.float64) for i in ref.control.generate_I_matrix(H, B, 0.1, 3)]
    else:
        H = [f32(np.zeros(s)) for s in S]
        I = [f32(np.zeros((1, s))) for s in S]
    gamma = 16.0
    q_pi, G = ref.control.update_posterior_policies_inductive(
        policies, qs, A, B, C, E, pA, pB, A_deps, B_deps, I, gamma=gamma, inductive_epsilon=eps,
        use_param_info_gain=use_pig, use_inductive=cfg["ind"])
    action = np.asarray(ref.control.sample_policy(policies, q_pi))
    adf, ado = deps_arrays(A_deps)
    bdf, bdo = deps_arrays(B_deps)
    data = dict(S=np.array(S, np.int64), O=np.array(O, np.int64), U=np.array(U, np.int64),
                T=np.int64(T), A_dep_flat=adf, A_dep_offsets=ado, B_dep_flat=bdf, B_dep_offsets=bdo,
                policies=policies, E=E.astype(np.float32), gamma=np.float64(gamma), eps=np.float64(eps),
                use_param_info_gain=np.int64(use_pig), use_inductive=np.int64(cfg["ind"]),
                has_pA=np.int64(cfg["pA"]), has_pB=np.int64(cfg["pB"]),
                I_depths=np.array([i.shape[0] for i in I], np.int64),
                q_pi=np.asarray(q_pi, np.float64), G=np.asarray(G, np.float64), action=action.astype(np.int32),
                C_ndim=np.array([np.ndim(c) for c in C], np.int64))
    data.update(pack("A", [a.astype(np.float32) for a in A]))
    data.update(pack("B", [b.astype(np.float32) for b in B]))
    data.update(pack("C", [c.astype(np.float32) for c in C]))
    data.update(pack("qs", [q.astype(np.float32) for q in qs]))
    data.update(pack("I", [i.astype(np.float32) for i in I]))
    data.update(pack("H", H))
    if pA is not None:
        data.update(pack("pA", pA))
    if pB is not None:
        data.update(pack("pB", pB))
    return data


def main(ref_root):
    sys.path.insert(0, HERE)
    import refshim

    ref = refshim.load_reference(ref_root)
    for name, cfg in FPI_CASES.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make_fpi_case(ref, name, cfg))
        print("wrote", name)
    for name, cfg in EFE_CASES.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make_efe_case(ref, name, cfg))
        print("wrote", name)
    for name, cfg in EFE_EXTRA_CASES.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make_efe_extra_case(ref, name, cfg))
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
