"""Golden fixtures for out-of-range inputs, made by the reference's own code.

    python tests/golden/make_golden_edges.py /root/reference

* ``fpi_bad_obs`` / ``fpi_bad_obs_single``: observations outside [0, O_m).
  ``Agent.infer_states`` turns index observations into one-hot vectors with
  ``jax.nn.one_hot`` (``pymdp/agent.py:659-673``), which is all zeros for an
  out-of-range index, and runs ``algos.run_factorized_fpi`` with
  ``distr_obs=True``; the zero vector's log-likelihood tensordot
  (``pymdp/maths.py:233-235``) is 0, so that modality adds nothing. The
  posteriors here come from ``run_factorized_fpi`` on exactly those one-hot
  vectors (``refshim``'s ``one_hot`` compares against ``arange`` as JAX's does).
* ``efe_bad_action``: policies holding actions outside [0, U_f).
  ``compute_expected_state`` reads ``B_f[..., u_f]`` (``pymdp/control.py:386``);
  under JAX a negative index counts from the end and an out-of-bounds gather
  index is clamped to the array's bounds. NumPy would raise instead, so this
  script applies that indexing rule to the policy matrix before the reference
  sees it (``jnp_index``), runs ``update_posterior_policies`` on the result,
  and stores the ORIGINAL policies with the reference's G and q_pi.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import deps_arrays, dirichlet_cols, f32, pack  # noqa: E402


def jnp_index(u, U):
    """The element a JAX gather reads for index u on an axis of size U."""
    u = np.where(u < 0, u + U, u)
    return np.clip(u, 0, U - 1)


def make_fpi_bad_obs(ref, S, O, deps, obs, seed):
    rng = np.random.default_rng(seed)
    batch, M, F = obs.shape[0], len(O), len(S)
    A = [np.stack([dirichlet_cols(rng, (O[m],) + tuple(S[d] for d in deps[m]), 0.7) for _ in range(batch)])
         for m in range(M)]
    prior = [np.stack([dirichlet_cols(rng, (s,), 1.0) for _ in range(batch)]) for s in S]
    qs = [np.zeros((batch, s)) for s in S]
    for b in range(batch):
        o_vec = [np.asarray(ref.nn.one_hot(obs[b, m], O[m])) for m in range(M)]
        out = ref.algos.run_factorized_fpi([a[b] for a in A], o_vec, [p[b] for p in prior], deps, num_iter=16)
        for f in range(F):
            qs[f][b] = out[f]
    dep_flat, dep_offs = deps_arrays(deps)
    data = dict(S=np.array(S, np.int64), O=np.array(O, np.int64), A_dep_flat=dep_flat, A_dep_offsets=dep_offs,
                num_iter=np.int64(16), obs=obs.astype(np.int32))
    data.update(pack("A", [a.astype(np.float32) for a in A]))
    data.update(pack("prior", [p.astype(np.float32) for p in prior]))
    data.update(pack("qs", qs))
    return data


def make_efe_bad_action(ref, seed=31):
    rng = np.random.default_rng(seed)
    S, O, U, T = [3, 2, 4], [4, 3], [2, 1, 3], 2
    A_deps, B_deps = [[0, 1], [2, 0]], [[0], [1], [2, 1]]
    F, M = len(S), len(O)
    A = [dirichlet_cols(rng, (O[m],) + tuple(S[d] for d in A_deps[m]), 0.5) for m in range(M)]
    B = [dirichlet_cols(rng, (S[f],) + tuple(S[d] for d in B_deps[f]) + (U[f],), 0.5) for f in range(F)]
    C = [f32(rng.normal(size=O[m])) for m in range(M)]
    qs = [dirichlet_cols(rng, (s,), 1.0) for s in S]
    pol = np.asarray(ref.control.construct_policies(S, U, T)).astype(np.int32)
    bad = pol.copy()
    bad[1, 0, 0] = 7     # beyond U: clamps to U - 1
    bad[2, 1, 2] = -1    # counts from the end: U - 1
    bad[3, 0, 1] = -5    # below -U: clamps to 0
    bad[4, 1, 0] = 2     # == U: clamps to U - 1
    bad[5, :, 2] = 9
    U_arr = np.array(U)[None, None, :]
    seen = jnp_index(bad, U_arr).astype(np.int32)
    P = pol.shape[0]
    E = f32(np.ones(P) / P)
    gamma = 16.0
    q_pi, G = ref.control.update_posterior_policies(seen, qs, A, B, C, E, None, None, A_deps, B_deps, gamma=gamma)
    adf, ado = deps_arrays(A_deps)
    bdf, bdo = deps_arrays(B_deps)
    data = dict(S=np.array(S, np.int64), O=np.array(O, np.int64), U=np.array(U, np.int64), T=np.int64(T),
                A_dep_flat=adf, A_dep_offsets=ado, B_dep_flat=bdf, B_dep_offsets=bdo, policies=bad,
                policies_as_read=seen, E=E.astype(np.float32), gamma=np.float64(gamma),
                q_pi=np.asarray(q_pi, np.float64), G=np.asarray(G, np.float64),
                C_ndim=np.array([np.ndim(c) for c in C], np.int64))
    data.update(pack("A", [a.astype(np.float32) for a in A]))
    data.update(pack("B", [b.astype(np.float32) for b in B]))
    data.update(pack("C", [c.astype(np.float32) for c in C]))
    data.update(pack("qs", [q.astype(np.float32) for q in qs]))
    return data


def main(ref_root):
    import refshim

    ref = refshim.load_reference(ref_root)
    import jax  # the shim's stand-in module, installed by load_reference

    ref.nn = jax.nn
    obs = np.array([[1, 2, 0, 5], [-1, 2, 3, 0], [4, 3, 1, 99], [-3, 7, 4, 6]], np.int32)
    cases = {
        "fpi_bad_obs": make_fpi_bad_obs(ref, [4, 3, 5], [5, 3, 4, 6], [[0, 1], [2], [1, 2], [0, 2]], obs, 41),
        "fpi_bad_obs_single": make_fpi_bad_obs(ref, [6], [4, 3], [[0], [0]],
                                               np.array([[3, 1], [4, 0], [-1, 2], [2, 3]], np.int32), 42),
        "efe_bad_action": make_efe_bad_action(ref),
    }
    for name, data in cases.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
