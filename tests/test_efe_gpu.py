"""EFE parity on the GPU: neg-EFE (G), q_pi and the selected action from the
sm_100a kernels (through the C-ABI) against golden vectors made by the
reference's own code (pymdp/control.py) and against the FP64 oracle.

Tolerance (FP32 and 3xTF32 paths vs FP64 reference): G rtol 1e-5 / atol
1e-5; q_pi within 1e-5 absolute (a probability vector: gamma = 16 turns an
absolute G error d into a relative q_pi error of 16 d, so a relative bound on
small entries would ask for G below FP32 resolution); selected actions
identical. BF16 path: G within 1e-3 of max(1, max |G|)."""

import numpy as np
import pytest
import torch

from conftest import deps_from, load_golden, unpack
from oracle import efe as oefe

pytestmark = pytest.mark.gpu

G_RTOL, G_ATOL = 1e-5, 1e-5
Q_RTOL, Q_ATOL = 0.0, 1e-5
EFE = ["efe_plain", "efe_mixed", "efe_bdeps", "efe_cfg3_t1", "efe_cfg3_small"]


def cuda(x, dtype=torch.float32):
    return torch.as_tensor(np.asarray(x), device="cuda").to(dtype)


def run_golden(d, precision="fp32"):
    from pymdp_b200 import ffi
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    qs = [cuda(q) for q in unpack(d, "qs")]
    I = [torch.zeros((1, q.shape[0]), device="cuda") for q in qs]
    G = ffi.neg_efe_all_policies_ffi(d["policies"], qs, [cuda(a) for a in unpack(d, "A")],
                                     [cuda(b) for b in unpack(d, "B")], [cuda(c) for c in unpack(d, "C")], I,
                                     A_deps, B_deps, use_inductive=False, precision=precision)
    q_pi = ffi.policy_posterior(G, cuda(d["E"]), float(d["gamma"]))
    act = ffi.select_action(q_pi, d["policies"])
    return G.cpu().numpy(), q_pi.cpu().numpy(), act.cpu().numpy()


@pytest.mark.parametrize("name", EFE)
def test_neg_efe_matches_reference(name):
    d = load_golden(name)
    G, q_pi, act = run_golden(d)
    np.testing.assert_allclose(G, d["G"], rtol=G_RTOL, atol=G_ATOL)
    np.testing.assert_allclose(q_pi, d["q_pi"], rtol=Q_RTOL, atol=Q_ATOL)
    np.testing.assert_array_equal(act, d["action"])


def random_efe(rng, S, O, U, T, A_deps, B_deps, batch, C2d=False):
    def dirc(shape, alpha=0.5):
        g = rng.gamma(alpha, size=shape) + 1e-30
        return (g / g.sum(1, keepdims=True)).astype(np.float32)
    A = [dirc((batch, O[m]) + tuple(S[d] for d in A_deps[m])) for m in range(len(O))]
    B = [dirc((batch, S[f]) + tuple(S[d] for d in B_deps[f]) + (U[f],)) for f in range(len(S))]
    C = [rng.normal(size=(batch, T, o) if C2d else (batch, o)).astype(np.float32) for o in O]
    qs = [dirc((batch, s), 1.0) for s in S]
    return A, B, C, qs


@pytest.mark.parametrize("case", [
    dict(S=[3, 4, 2], O=[4, 5, 3], U=[2, 3, 2], T=2, A_deps=[[0, 2], [1, 2, 0], [1]], B_deps=[[0], [1, 0], [2, 1]]),
    dict(S=[5, 3], O=[7], U=[3, 2], T=3, A_deps=[[1, 0]], B_deps=[[0], [1]], C2d=True),
    dict(S=[2, 2, 2, 2], O=[3, 3], U=[2, 1, 2, 1], T=2, A_deps=[[0, 1, 2, 3], [3, 1]],
         B_deps=[[0], [1], [2, 3], [3]]),
    dict(S=[6], O=[4, 2], U=[5], T=1, A_deps=[[0], [0]], B_deps=[[0]]),
])
@pytest.mark.parametrize("flags", [(True, True), (True, False), (False, True), (False, False)])
def test_neg_efe_random_models_match_oracle(case, flags):
    from pymdp_b200 import ffi
    rng = np.random.default_rng(len(case["S"]) * 7 + case["T"])
    batch = 3
    A, B, C, qs = random_efe(rng, case["S"], case["O"], case["U"], case["T"], case["A_deps"], case["B_deps"],
                             batch, case.get("C2d", False))
    pol = oefe.construct_policies(case["S"], case["U"], case["T"])
    I = [torch.zeros((batch, 1, s), device="cuda") for s in case["S"]]
    G = ffi.neg_efe_all_policies_ffi(pol, [cuda(q) for q in qs], [cuda(a) for a in A], [cuda(b) for b in B],
                                     [cuda(c) for c in C], I, case["A_deps"], case["B_deps"], use_utility=flags[0],
                                     use_states_info_gain=flags[1], use_inductive=False).cpu().numpy()
    for b in range(batch):
        ref = oefe.neg_efe_all_policies(pol, [q[b] for q in qs], [a[b] for a in A], [x[b] for x in B],
                                        [c[b] for c in C], case["A_deps"], case["B_deps"], use_utility=flags[0],
                                        use_states_info_gain=flags[1])
        np.testing.assert_allclose(G[b], ref, rtol=G_RTOL, atol=G_ATOL)


@pytest.mark.parametrize("precision", ["fp32", "tf32x3", "bf16"])
def test_out_of_range_action_reads_b_as_jax_indexing_does(precision):
    """Actions outside [0, U_f) index B_f[..., u] as jnp indexing does
    (negative from the end, then clamped): G and q_pi equal the reference's
    on the clamped policies (tests/golden/make_golden_edges.py)."""
    from pymdp_b200 import ffi
    d = load_golden("efe_bad_action")
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    qs = [cuda(q) for q in unpack(d, "qs")]
    I = [torch.zeros((1, q.shape[0]), device="cuda") for q in qs]
    G = ffi.neg_efe_all_policies_ffi(d["policies"], qs, [cuda(a) for a in unpack(d, "A")],
                                     [cuda(b) for b in unpack(d, "B")], [cuda(c) for c in unpack(d, "C")], I,
                                     A_deps, B_deps, use_inductive=False, precision=precision)
    q_pi = ffi.policy_posterior(G, cuda(d["E"]), float(d["gamma"])).cpu().numpy().reshape(-1)
    G = G.cpu().numpy().reshape(-1)
    assert np.isfinite(G).all()
    _g_close(G, d["G"], precision)
    if precision != "bf16":
        np.testing.assert_allclose(q_pi, d["q_pi"], rtol=Q_RTOL, atol=Q_ATOL)


# ---------------------------------------------------------- tensor-core paths
# TF32x3 (tcgen05 kind::tf32, hi/lo split) is held to the FP32 tolerance; the
# 3-pass BF16 split (kind::f16) to the BF16 tier: G within 1e-3 of max(1, |G|).
TC_TOL = {"fp32": (G_RTOL, G_ATOL), "tf32x3": (G_RTOL, G_ATOL), "bf16": (0.0, 1e-3)}


def _g_close(G, ref, precision):
    rtol, atol = TC_TOL[precision]
    if precision == "bf16":
        scale = np.maximum(np.abs(ref).max(), 1.0)
        np.testing.assert_allclose(G, ref, rtol=0, atol=atol * scale)
    else:
        np.testing.assert_allclose(G, ref, rtol=rtol, atol=atol)


@pytest.mark.parametrize("precision", ["tf32x3", "bf16"])
@pytest.mark.parametrize("name", EFE)
def test_tensor_core_neg_efe_matches_reference(name, precision):
    from pymdp_b200 import _lib
    d = load_golden(name)
    G, q_pi, act = run_golden(d, precision)
    assert _lib.load().b2_device_error() == 0
    _g_close(G, d["G"], precision)
    if precision == "tf32x3":
        np.testing.assert_allclose(q_pi, d["q_pi"], rtol=Q_RTOL, atol=Q_ATOL)
        np.testing.assert_array_equal(act, d["action"])


@pytest.mark.parametrize("precision", ["tf32x3", "bf16"])
@pytest.mark.parametrize("case", [
    dict(S=[3, 4, 2], O=[4, 5, 3], U=[2, 3, 2], T=2, A_deps=[[0, 2], [1, 2, 0], [1]], B_deps=[[0], [1, 0], [2, 1]]),
    dict(S=[5, 3], O=[7], U=[3, 2], T=3, A_deps=[[1, 0]], B_deps=[[0], [1]], C2d=True),
    dict(S=[9, 7, 5], O=[11, 3, 6], U=[4, 3, 1], T=2, A_deps=[[0, 1, 2], [0, 1, 2], [2, 0]], B_deps=[[0], [1], [2]]),
    dict(S=[32, 16, 8], O=[16, 16, 8, 8, 4], U=[4, 4, 1], T=2, A_deps=[[0, 1, 2]] * 5, B_deps=[[0], [1], [2]]),
])
def test_tensor_core_random_models_match_oracle(case, precision):
    from pymdp_b200 import _lib, ffi
    rng = np.random.default_rng(len(case["S"]) * 11 + case["T"])
    batch = 2
    A, B, C, qs = random_efe(rng, case["S"], case["O"], case["U"], case["T"], case["A_deps"], case["B_deps"],
                             batch, case.get("C2d", False))
    pol = oefe.construct_policies(case["S"], case["U"], case["T"])
    I = [torch.zeros((batch, 1, s), device="cuda") for s in case["S"]]
    G = ffi.neg_efe_all_policies_ffi(pol, [cuda(q) for q in qs], [cuda(a) for a in A], [cuda(b) for b in B],
                                     [cuda(c) for c in C], I, case["A_deps"], case["B_deps"], use_inductive=False,
                                     precision=precision).cpu().numpy()
    assert _lib.load().b2_device_error() == 0
    for b in range(batch):
        ref = oefe.neg_efe_all_policies(pol, [q[b] for q in qs], [a[b] for a in A], [x[b] for x in B],
                                        [c[b] for c in C], case["A_deps"], case["B_deps"])
        _g_close(G[b], ref, precision)


# ------------------------------------------- flag-gated terms (bits 2 and 3)
# Parameter information gain (pA / pB, exact Dirichlet weight with digamma)
# and the inductive value, against golden vectors from the reference's
# update_posterior_policies_inductive (pymdp/control.py:795-963) and against
# the FP64 oracle on random models. These terms run on the FP32 SIMT kernel
# for every precision selector, so the FP32 tolerance applies to all three.
EFE_EXTRA = ["efe_pig", "efe_pigA", "efe_ind", "efe_all"]


def run_golden_extra(d, precision):
    from pymdp_b200 import ffi
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    qs = [cuda(q) for q in unpack(d, "qs")]
    pA = [cuda(a) for a in unpack(d, "pA")] if int(d["has_pA"]) else None
    pB = [cuda(b) for b in unpack(d, "pB")] if int(d["has_pB"]) else None
    G = ffi.neg_efe_all_policies_ffi(d["policies"], qs, [cuda(a) for a in unpack(d, "A")],
                                     [cuda(b) for b in unpack(d, "B")], [cuda(c) for c in unpack(d, "C")],
                                     [cuda(i) for i in unpack(d, "I")], A_deps, B_deps, pA=pA, pB=pB,
                                     use_param_info_gain=bool(int(d["use_param_info_gain"])),
                                     use_inductive=bool(int(d["use_inductive"])),
                                     inductive_epsilon=float(d["eps"]), precision=precision)
    q_pi = ffi.policy_posterior(G, cuda(d["E"]), float(d["gamma"]))
    act = ffi.select_action(q_pi, d["policies"])
    return G.cpu().numpy(), q_pi.cpu().numpy(), act.cpu().numpy()


@pytest.mark.parametrize("precision", ["fp32", "tf32x3", "bf16"])
@pytest.mark.parametrize("name", EFE_EXTRA)
def test_flag_gated_terms_match_reference(name, precision):
    d = load_golden(name)
    G, q_pi, act = run_golden_extra(d, precision)
    np.testing.assert_allclose(G, d["G"], rtol=G_RTOL, atol=G_ATOL)
    np.testing.assert_allclose(q_pi, d["q_pi"], rtol=Q_RTOL, atol=Q_ATOL)
    np.testing.assert_array_equal(act, d["action"])


@pytest.mark.parametrize("terms", ["pA", "pB", "pApB", "ind", "all"])
def test_flag_gated_terms_random_models_match_oracle(terms):
    from pymdp_b200 import ffi
    S, O, U, T = [4, 3, 2], [5, 3], [3, 2, 2], 2
    A_deps, B_deps = [[0, 2], [1, 0]], [[0], [1, 0], [2]]
    rng = np.random.default_rng(len(terms) + 31)
    batch = 3
    A, B, C, qs = random_efe(rng, S, O, U, T, A_deps, B_deps, batch)
    counts = lambda shape: (rng.gamma(1.5, size=shape) * 2 * (rng.random(size=shape) > 0.1)).astype(np.float32)
    pA = [counts(a.shape) for a in A] if "pA" in terms or terms == "all" else None
    pB = [counts(b.shape) for b in B] if "pB" in terms or terms == "all" else None
    use_ind = terms in ("ind", "all")
    I = [(rng.random(size=(batch, 3, s)) > 0.5).astype(np.float32) for s in S]
    eps = np.array([1e-3, 1e-2, 0.2], np.float32)
    pol = oefe.construct_policies(S, U, T)
    G = ffi.neg_efe_all_policies_ffi(pol, [cuda(q) for q in qs], [cuda(a) for a in A], [cuda(b) for b in B],
                                     [cuda(c) for c in C], [cuda(i) for i in I], A_deps, B_deps,
                                     pA=[cuda(x) for x in pA] if pA else None,
                                     pB=[cuda(x) for x in pB] if pB else None,
                                     use_param_info_gain=pA is not None or pB is not None, use_inductive=use_ind,
                                     inductive_epsilon=cuda(eps)).cpu().numpy()
    for b in range(batch):
        ref = oefe.neg_efe_all_policies(pol, [q[b] for q in qs], [a[b] for a in A], [x[b] for x in B],
                                        [c[b] for c in C], A_deps, B_deps,
                                        pA=[x[b] for x in pA] if pA else None,
                                        pB=[x[b] for x in pB] if pB else None,
                                        use_param_info_gain=pA is not None or pB is not None,
                                        I=[i[b] for i in I], use_inductive=use_ind,
                                        inductive_epsilon=float(eps[b]))
        np.testing.assert_allclose(G[b], ref, rtol=G_RTOL, atol=G_ATOL * max(1.0, np.abs(ref).max()))


def test_agent_with_param_info_gain_and_inductive_matches_oracle():
    """The Agent facade with pA, pB and goal vectors H (I built by
    generate_I_matrix, pymdp/agent.py:368-380) against the FP64 oracle."""
    from pymdp_b200 import Agent
    from pymdp_b200.control import generate_I_matrix
    S, O, U, T = [4, 3], [5, 3], [3, 2], 2
    A_deps, B_deps = [[0, 1], [1]], [[0], [1]]
    rng = np.random.default_rng(77)
    batch = 2
    A, B, C, qs = random_efe(rng, S, O, U, T, A_deps, B_deps, batch)
    pA = [(rng.gamma(2.0, size=a.shape) * 2).astype(np.float32) for a in A]
    pB = [(rng.gamma(2.0, size=b.shape) * 2).astype(np.float32) for b in B]
    H = [np.eye(s, dtype=np.float32)[s - 1] for s in S]
    agent = Agent(A, B, C=C, A_dependencies=A_deps, B_dependencies=B_deps, policy_len=T, gamma=16.0,
                  batch_size=batch, pA=pA, pB=pB, H=H, inductive_depth=3, inductive_threshold=0.1,
                  inductive_epsilon=1e-3, use_param_info_gain=True, use_inductive=True)
    q_pi, G = agent.infer_policies([cuda(q) for q in qs])
    pol = oefe.construct_policies(S, U, T)
    for b in range(batch):
        I = generate_I_matrix(H, [x[b] for x in B], 0.1, 3)
        E = np.full(len(pol), 1.0 / len(pol))
        q_ref, G_ref = oefe.update_posterior_policies(
            pol, [q[b] for q in qs], [a[b] for a in A], [x[b] for x in B], [c[b] for c in C], E, A_deps, B_deps,
            gamma=16.0, pA=[x[b] for x in pA], pB=[x[b] for x in pB], use_param_info_gain=True, I=I,
            use_inductive=True, inductive_epsilon=1e-3)
        np.testing.assert_allclose(G[b].cpu().numpy(), G_ref, rtol=G_RTOL, atol=G_ATOL * max(1.0, np.abs(G_ref).max()))
        np.testing.assert_allclose(q_pi[b].cpu().numpy(), q_ref, rtol=Q_RTOL, atol=Q_ATOL)


# ----------------------------------------- policy-tree mode (B2_FLAG_POLICY_TREE)
@pytest.mark.parametrize("precision", ["tf32x3", "bf16"])
@pytest.mark.parametrize("case", [
    dict(S=[3, 4, 2], O=[4, 5, 3], U=[2, 3, 2], T=2, A_deps=[[0, 2], [1, 2, 0], [1]], B_deps=[[0], [1, 0], [2, 1]]),
    dict(S=[5, 3], O=[7], U=[3, 2], T=3, A_deps=[[1, 0]], B_deps=[[0], [1]], C2d=True),
    dict(S=[32, 16, 8], O=[16, 16, 8, 8, 4], U=[4, 4, 1], T=3, A_deps=[[0, 1, 2]] * 5, B_deps=[[0], [1], [2]]),
])
def test_policy_tree_matches_oracle_and_full_evaluation(case, precision):
    """Evaluating each distinct policy prefix once (T >= 2, the full product
    policy set) gives the oracle's G, and the per-policy evaluation's."""
    from pymdp_b200 import _lib, ffi
    rng = np.random.default_rng(len(case["S"]) * 7 + case["T"])
    batch = 2
    A, B, C, qs = random_efe(rng, case["S"], case["O"], case["U"], case["T"], case["A_deps"], case["B_deps"],
                             batch, case.get("C2d", False))
    pol = oefe.construct_policies(case["S"], case["U"], case["T"])
    I = [torch.zeros((batch, 1, s), device="cuda") for s in case["S"]]
    args = (pol, [cuda(q) for q in qs], [cuda(a) for a in A], [cuda(b) for b in B], [cuda(c) for c in C], I,
            case["A_deps"], case["B_deps"])
    G_tree = ffi.neg_efe_all_policies_ffi(*args, use_inductive=False, precision=precision,
                                          policy_tree=True).cpu().numpy()
    G_full = ffi.neg_efe_all_policies_ffi(*args, use_inductive=False, precision=precision).cpu().numpy()
    assert _lib.load().b2_device_error() == 0
    for b in range(batch):
        ref = oefe.neg_efe_all_policies(pol, [q[b] for q in qs], [a[b] for a in A], [x[b] for x in B],
                                        [c[b] for c in C], case["A_deps"], case["B_deps"])
        _g_close(G_tree[b], ref, precision)
        _g_close(G_full[b], ref, precision)


@pytest.mark.parametrize("precision", ["tf32x3", "bf16"])
def test_pack_cache_reuses_operand_images(precision):
    """b2_neg_efe_cached: the first call packs (and sets the valid flag), the
    second reuses the images; both equal b2_neg_efe bit for bit. Clearing the
    flag after A changes repacks."""
    import ctypes
    from pymdp_b200 import ffi
    case = dict(S=[9, 7, 5], O=[11, 3, 6], U=[4, 3, 1], T=2, A_deps=[[0, 1, 2], [0, 1, 2], [2, 0]],
                B_deps=[[0], [1], [2]])
    rng = np.random.default_rng(5)
    batch = 3
    A, B, C, qs = random_efe(rng, case["S"], case["O"], case["U"], case["T"], case["A_deps"], case["B_deps"], batch)
    pol = torch.as_tensor(oefe.construct_policies(case["S"], case["U"], case["T"]), device="cuda").int().contiguous()
    P = pol.shape[0]
    lay = ffi.EfeLayout(case["S"], case["O"], case["U"], case["T"], case["A_deps"], case["B_deps"])
    flat = lambda xs: ffi.flatten_ragged_f32([cuda(x) for x in xs], 1)[0]  # noqa: E731
    qs_f, A_f, B_f, C_f = flat(qs), flat(A), flat(B), flat([np.repeat(c[:, None, :], case["T"], 1) for c in C])
    I_f = torch.zeros((batch, int(lay.I_offsets[-1])), device="cuda")
    eps = torch.full((1,), 1e-3, device="cuda")
    flags = ffi.efe_flags(precision=precision, policy_tree=True)

    def run(cache=None):
        out = torch.empty((batch, P), device="cuda")
        lay.call(None, pol, 0, qs_f, A_f, B_f, C_f, I_f, None, None, eps, out, batch, P, flags, cache=cache)
        return out.cpu().numpy()

    n = lay.pack_bytes(batch, P, flags)
    assert n > 0
    cache = (torch.empty(n, dtype=torch.uint8, device="cuda"), ctypes.c_int32(0))
    ref = run()
    first = run(cache)
    assert cache[1].value == 1
    second = run(cache)
    np.testing.assert_array_equal(first, ref)
    np.testing.assert_array_equal(second, ref)
    A_f.mul_(0.5).add_(0.5 / 11)  # a different (still normalised for modality 0) A: repack
    cache[1].value = 0
    np.testing.assert_array_equal(run(cache), run())


# ------------------------------------------------ action selection modes
def _random_qpi(rng, batch, P, alpha=2.0):
    g = rng.gamma(alpha, size=(batch, P))
    return (g / g.sum(1, keepdims=True)).astype(np.float32)


def test_sample_action_modes_match_oracle():
    """b2_sample_action: deterministic "full" and "marginal" equal the
    reference's argmax rules; stochastic draws equal the oracle's restatement
    of the same Gumbel-max draw (except where the perturbed logits tie within
    1e-4)."""
    from pymdp_b200 import ffi
    rng = np.random.default_rng(21)
    U, T, batch, alpha, seed = [3, 2, 1], 2, 64, 3.0, 1234
    pol = oefe.construct_policies([3, 2, 2], U, T)
    q = _random_qpi(rng, batch, len(pol))
    qd = cuda(q)
    full_det = ffi.sample_action(qd, pol, U, "full", "deterministic").cpu().numpy()
    marg_det = ffi.sample_action(qd, pol, U, "marginal", "deterministic").cpu().numpy()
    full_sto = ffi.sample_action(qd, pol, U, "full", "stochastic", alpha, seed).cpu().numpy()
    marg_sto = ffi.sample_action(qd, pol, U, "marginal", "stochastic", alpha, seed).cpu().numpy()
    ties = 0
    for b in range(batch):
        np.testing.assert_array_equal(full_det[b], oefe.sample_policy(pol, q[b]))
        np.testing.assert_array_equal(marg_det[b], oefe.sample_action_marginal(pol, U, q[b]))
        p, gap = oefe.sample_stochastic(q[b], alpha, seed, b, -1)
        if gap > 1e-4:
            np.testing.assert_array_equal(full_sto[b], pol[p, 0])
        else:
            ties += 1
        for f, m in enumerate(oefe.get_marginals(q[b], pol, U)):
            a, gap = oefe.sample_stochastic(m, alpha, seed, b, f)
            if gap > 1e-4:
                assert marg_sto[b, f] == a, (b, f)
    assert ties <= 1


@pytest.mark.parametrize("mode", ["full", "marginal"])
@pytest.mark.parametrize("alpha", [1.0, 4.0])
def test_stochastic_selection_follows_the_softmax(mode, alpha):
    """Stochastic draws across many agents with the same q_pi follow
    softmax(alpha * log q) (total variation below 0.015 over 40000 draws)."""
    from pymdp_b200 import ffi
    U, T, batch = [6], 1, 40000
    pol = oefe.construct_policies([6], U, T)
    q1 = np.array([0.05, 0.1, 0.15, 0.2, 0.22, 0.28], np.float32)
    q = np.broadcast_to(q1, (batch, 6)).copy()
    act = ffi.sample_action(cuda(q), pol, U, mode, "stochastic", alpha, 99).cpu().numpy()[:, 0]
    freq = np.bincount(act, minlength=6) / batch
    p = np.exp(alpha * np.log(q1.astype(np.float64)))
    p /= p.sum()
    assert 0.5 * np.abs(freq - p).sum() < 0.015, (freq, p)


def test_agent_stochastic_marginal_mode_runs():
    from pymdp_b200 import Agent
    rng = np.random.default_rng(3)
    A = [rng.dirichlet(np.ones(3), size=(3, 2)).transpose(2, 0, 1).astype(np.float32)]
    B = [rng.dirichlet(np.ones(3), size=(3, 3)).transpose(2, 0, 1).astype(np.float32),
         rng.dirichlet(np.ones(2), size=(2, 2)).transpose(2, 0, 1).astype(np.float32)]
    agent = Agent(A, B, policy_len=2, batch_size=5, alpha=8.0, action_selection="stochastic",
                  sampling_mode="marginal")
    qs = agent.infer_states(torch.zeros((5, 1), dtype=torch.int32, device="cuda"),
                            [torch.full((5, 3), 1 / 3, device="cuda"), torch.full((5, 2), 0.5, device="cuda")])
    q_pi, _ = agent.infer_policies(qs)
    with pytest.raises(ValueError):
        agent.sample_action(q_pi)
    act = agent.sample_action(q_pi, rng_key=7).cpu().numpy()
    assert act.shape == (5, 2) and (act[:, 0] < 3).all() and (act[:, 1] < 2).all()


@pytest.mark.parametrize("efe_algorithm,precision", [("dense", "tf32x3"), ("factored", "fp32")])
def test_full_benchmark_model_within_1e5(efe_algorithm, precision):
    """The EFE benchmark model at full size, as the Agent runs it (3xTF32 tensor
    cores in policy-tree mode with the pack cache, or the factored path): S=[32,16,8], U=[4,4,1], T=3 (4096 policies),
    O=[16,16,8,8,4] on all factors, A, B ~ Dirichlet(0.5), C ~ N(0,1), 8
    agents with FPI posteriors as beliefs. Every G within 1e-5 relative of the
    FP64 oracle (floor 1e-6, the bench's criterion), q_pi within 1e-5 absolute,
    actions identical."""
    import bench
    from pymdp_b200 import Agent, _lib
    n = 8
    A, B, C, D, obs = bench.make_model(4321, n)
    agent = Agent(A, B, C=C, D=D, policy_len=bench.T, gamma=bench.GAMMA, batch_size=n, num_iter=16,
                  precision=precision, efe_algorithm=efe_algorithm)
    qs = agent.infer_states(torch.as_tensor(obs, device="cuda"), [cuda(d) for d in D])
    q_pi, G = agent.infer_policies(qs)
    act = agent.sample_action(q_pi).cpu().numpy()
    assert _lib.load().b2_device_error() == 0
    G, q_pi = G.cpu().numpy().astype(np.float64), q_pi.cpu().numpy()
    pol = oefe.construct_policies(bench.S, bench.U, bench.T)
    E = np.full(len(pol), 1.0 / len(pol))
    worst = 0.0
    for b in range(n):
        q32 = [q[b, 0].cpu().numpy().astype(np.float64) for q in qs]
        q_ref, G_ref = oefe.update_posterior_policies(pol, q32, [a[b] for a in A], [x[b] for x in B],
                                                      [c[b] for c in C], E, [[0, 1, 2]] * 5, [[0], [1], [2]],
                                                      gamma=bench.GAMMA)
        worst = max(worst, float(np.max(np.abs(G[b] - G_ref) / np.maximum(np.abs(G_ref), 1e-6))))
        np.testing.assert_allclose(q_pi[b], q_ref, rtol=0, atol=1e-5)
        np.testing.assert_array_equal(act[b], oefe.sample_policy(pol, q_ref))
    assert worst <= 1e-5, worst


# ------------------------------------------------ factored path (B2_FLAG_FACTORED)
FACT_CASES = [
    # the benchmark family at T = 3 (one rank-3 group), few agents
    dict(S=[32, 16, 8], O=[16, 16, 8, 8, 4], U=[4, 4, 1], T=3, A_deps=[[0, 1, 2]] * 5, B_deps=[[0], [1], [2]]),
    # groups of rank 1, 2 and 3 with permuted dependency order, every factor controllable
    dict(S=[3, 4, 2], O=[4, 5, 3], U=[2, 3, 2], T=2, A_deps=[[0, 2], [1, 2, 0], [1]], B_deps=[[0], [1], [2]]),
    # time-indexed C, horizon 3
    dict(S=[5, 3], O=[7, 2], U=[3, 2], T=3, A_deps=[[1, 0], [0]], B_deps=[[0], [1]], C2d=True),
    # horizon 1 (no tree levels below the root), an uncontrolled factor
    dict(S=[6, 4, 3], O=[4, 2], U=[5, 1, 2], T=1, A_deps=[[0, 1], [2, 1, 0]], B_deps=[[0], [1], [2]]),
    # a factor no modality observes
    dict(S=[4, 3, 5], O=[6], U=[2, 2, 3], T=2, A_deps=[[2, 0]], B_deps=[[0], [1], [2]]),
    # 101 observation rows: the tail's level-2 tile falls back to 8 histories (16 would not fit shared memory)
    dict(S=[16, 16, 16], O=[60, 41], U=[2, 2, 2], T=2, A_deps=[[0, 1, 2]] * 2, B_deps=[[0], [1], [2]]),
]


@pytest.mark.parametrize("flags", [(True, True), (True, False), (False, True)])
@pytest.mark.parametrize("ci", range(len(FACT_CASES)))
def test_factored_neg_efe_matches_oracle(ci, flags):
    """B2_FLAG_FACTORED: the contraction factor by factor over the per-factor
    history marginals gives the FP64 oracle's G (FP32 tolerance)."""
    from pymdp_b200 import _lib, ffi
    case = FACT_CASES[ci]
    rng = np.random.default_rng(100 + ci)
    batch = 2
    A, B, C, qs = random_efe(rng, case["S"], case["O"], case["U"], case["T"], case["A_deps"], case["B_deps"],
                             batch, case.get("C2d", False))
    pol = oefe.construct_policies(case["S"], case["U"], case["T"])
    I = [torch.zeros((batch, 1, s), device="cuda") for s in case["S"]]
    n0 = _lib.launch_count()
    G = ffi.neg_efe_all_policies_ffi(pol, [cuda(q) for q in qs], [cuda(a) for a in A], [cuda(b) for b in B],
                                     [cuda(c) for c in C], I, case["A_deps"], case["B_deps"], use_utility=flags[0],
                                     use_states_info_gain=flags[1], use_inductive=False, policy_tree=True,
                                     factored=True).cpu().numpy()
    assert _lib.launch_count() - n0 == 4  # histories, level 1, tail, combine
    for b in range(batch):
        ref = oefe.neg_efe_all_policies(pol, [q[b] for q in qs], [a[b] for a in A], [x[b] for x in B],
                                        [c[b] for c in C], case["A_deps"], case["B_deps"], use_utility=flags[0],
                                        use_states_info_gain=flags[1])
        np.testing.assert_allclose(G[b], ref, rtol=G_RTOL, atol=G_ATOL)


@pytest.mark.parametrize("case", [
    # multi-parent transitions: not factor-local
    dict(S=[3, 4, 2], O=[4, 5], U=[2, 3, 2], T=2, A_deps=[[0, 2], [1, 2, 0]], B_deps=[[0], [1, 0], [2, 1]]),
    # a rank-4 dependency tuple
    dict(S=[2, 2, 2, 2], O=[3, 3], U=[2, 1, 2, 1], T=2, A_deps=[[0, 1, 2, 3], [3, 1]], B_deps=[[0], [1], [2], [3]]),
])
def test_factored_flag_outside_its_conditions_takes_another_path(case):
    """Where the factored contraction does not apply, the flag is ignored and
    the result still equals the oracle's."""
    from pymdp_b200 import _lib, ffi
    rng = np.random.default_rng(7)
    batch = 2
    A, B, C, qs = random_efe(rng, case["S"], case["O"], case["U"], case["T"], case["A_deps"], case["B_deps"], batch)
    pol = oefe.construct_policies(case["S"], case["U"], case["T"])
    I = [torch.zeros((batch, 1, s), device="cuda") for s in case["S"]]
    n0 = _lib.launch_count()
    G = ffi.neg_efe_all_policies_ffi(pol, [cuda(q) for q in qs], [cuda(a) for a in A], [cuda(b) for b in B],
                                     [cuda(c) for c in C], I, case["A_deps"], case["B_deps"], use_inductive=False,
                                     policy_tree=True, factored=True).cpu().numpy()
    assert _lib.launch_count() - n0 != 4
    for b in range(batch):
        ref = oefe.neg_efe_all_policies(pol, [q[b] for q in qs], [a[b] for a in A], [x[b] for x in B],
                                        [c[b] for c in C], case["A_deps"], case["B_deps"])
        np.testing.assert_allclose(G[b], ref, rtol=G_RTOL, atol=G_ATOL)


@pytest.mark.parametrize("name", ["efe_plain", "efe_mixed", "efe_cfg3_t1", "efe_cfg3_small"])
def test_factored_neg_efe_matches_reference(name):
    """The factored path on the golden fixtures whose transitions are factor-local."""
    from pymdp_b200 import ffi
    d = load_golden(name)
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    qs = [cuda(q) for q in unpack(d, "qs")]
    I = [torch.zeros((1, q.shape[0]), device="cuda") for q in qs]
    G = ffi.neg_efe_all_policies_ffi(d["policies"], qs, [cuda(a) for a in unpack(d, "A")],
                                     [cuda(b) for b in unpack(d, "B")], [cuda(c) for c in unpack(d, "C")], I,
                                     A_deps, B_deps, use_inductive=False, policy_tree=True, factored=True)
    q_pi = ffi.policy_posterior(G, cuda(d["E"]), float(d["gamma"]))
    act = ffi.select_action(q_pi, d["policies"])
    np.testing.assert_allclose(G.cpu().numpy(), d["G"], rtol=G_RTOL, atol=G_ATOL)
    np.testing.assert_allclose(q_pi.cpu().numpy(), d["q_pi"], rtol=Q_RTOL, atol=Q_ATOL)
    np.testing.assert_array_equal(act.cpu().numpy(), d["action"])


@pytest.mark.parametrize("name", ["efe_pigA", "efe_ind", "efe_all"])
def test_factored_flag_gated_terms_match_reference(name):
    """Parameter information gain (pA rows carried through the factored
    contraction, pB per factor history) and the inductive value on the
    factored path, against the reference's update_posterior_policies_inductive
    fixtures (factor-local transitions)."""
    from pymdp_b200 import _lib, ffi
    d = load_golden(name)
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    assert all(b == [f] for f, b in enumerate(B_deps))
    qs = [cuda(q) for q in unpack(d, "qs")]
    pA = [cuda(a) for a in unpack(d, "pA")] if int(d["has_pA"]) else None
    pB = [cuda(b) for b in unpack(d, "pB")] if int(d["has_pB"]) else None
    n0 = _lib.launch_count()
    G = ffi.neg_efe_all_policies_ffi(d["policies"], qs, [cuda(a) for a in unpack(d, "A")],
                                     [cuda(b) for b in unpack(d, "B")], [cuda(c) for c in unpack(d, "C")],
                                     [cuda(i) for i in unpack(d, "I")], A_deps, B_deps, pA=pA, pB=pB,
                                     use_param_info_gain=bool(int(d["use_param_info_gain"])),
                                     use_inductive=bool(int(d["use_inductive"])),
                                     inductive_epsilon=float(d["eps"]), policy_tree=True, factored=True)
    launches = _lib.launch_count() - n0
    q_pi = ffi.policy_posterior(G, cuda(d["E"]), float(d["gamma"]))
    act = ffi.select_action(q_pi, d["policies"])
    weights = int(pA is not None) + int(pB is not None) + int(bool(int(d["use_inductive"])))
    assert launches == 4 + weights  # the weight kernels, then the factored path's four
    np.testing.assert_allclose(G.cpu().numpy(), d["G"], rtol=G_RTOL, atol=G_ATOL)
    np.testing.assert_allclose(q_pi.cpu().numpy(), d["q_pi"], rtol=Q_RTOL, atol=Q_ATOL)
    np.testing.assert_array_equal(act.cpu().numpy(), d["action"])


@pytest.mark.parametrize("terms", ["pA", "pB", "pApB", "ind", "all"])
def test_factored_flag_gated_terms_random_models_match_oracle(terms):
    from pymdp_b200 import ffi
    S, O, U, T = [4, 3, 2], [5, 3, 2], [3, 2, 2], 2
    A_deps, B_deps = [[0, 2], [1, 0], [2, 1, 0]], [[0], [1], [2]]
    rng = np.random.default_rng(len(terms) + 61)
    batch = 3
    A, B, C, qs = random_efe(rng, S, O, U, T, A_deps, B_deps, batch)
    counts = lambda shape: (rng.gamma(1.5, size=shape) * 2 * (rng.random(size=shape) > 0.1)).astype(np.float32)
    pA = [counts(a.shape) for a in A] if "pA" in terms or terms == "all" else None
    pB = [counts(b.shape) for b in B] if "pB" in terms or terms == "all" else None
    use_ind = terms in ("ind", "all")
    I = [(rng.random(size=(batch, 3, s)) > 0.5).astype(np.float32) for s in S]
    eps = np.array([1e-3, 1e-2, 0.2], np.float32)
    pol = oefe.construct_policies(S, U, T)
    G = ffi.neg_efe_all_policies_ffi(pol, [cuda(q) for q in qs], [cuda(a) for a in A], [cuda(b) for b in B],
                                     [cuda(c) for c in C], [cuda(i) for i in I], A_deps, B_deps,
                                     pA=[cuda(x) for x in pA] if pA else None,
                                     pB=[cuda(x) for x in pB] if pB else None,
                                     use_param_info_gain=pA is not None or pB is not None, use_inductive=use_ind,
                                     inductive_epsilon=cuda(eps), policy_tree=True, factored=True).cpu().numpy()
    for b in range(batch):
        ref = oefe.neg_efe_all_policies(pol, [q[b] for q in qs], [a[b] for a in A], [x[b] for x in B],
                                        [c[b] for c in C], A_deps, B_deps,
                                        pA=[x[b] for x in pA] if pA else None,
                                        pB=[x[b] for x in pB] if pB else None,
                                        use_param_info_gain=pA is not None or pB is not None,
                                        I=[i[b] for i in I], use_inductive=use_ind,
                                        inductive_epsilon=float(eps[b]))
        np.testing.assert_allclose(G[b], ref, rtol=G_RTOL, atol=G_ATOL * max(1.0, np.abs(ref).max()))
