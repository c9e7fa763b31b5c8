"""Online Dirichlet learning on the GPU through the C-ABI
(``b2_update_obs_likelihood_dirichlet``, ``b2_update_state_transition_dirichlet``)
against the golden fixtures made by the reference's ``pymdp/learning.py`` and
the FP64 oracle (``oracle/learning.py``).

Tolerances: pA / pB take one float32 multiply-add per observation
(rtol 2e-6); A / B are float32 quotients of float32 sums (rtol 2e-6,
atol 1e-7)."""

import numpy as np
import pytest
import torch

from conftest import load_golden, unpack
from oracle import efe as oefe
from oracle import learning as ol

pytestmark = pytest.mark.gpu

P_RTOL = 2e-6
E_RTOL, E_ATOL = 2e-6, 1e-7


def cuda(x, dtype=torch.float32):
    return torch.as_tensor(np.asarray(x), device="cuda").to(dtype).contiguous()


def _deps(d):
    out, i = [], 0
    for n in d["deps_len"]:
        out.append(d["deps_flat"][i:i + n].tolist())
        i += n
    return out


def flat(arrays, Bn):
    return cuda(np.concatenate([np.asarray(a).reshape(Bn, -1) for a in arrays], axis=1))


def split(t, shapes):
    out, o = [], 0
    x = t.cpu().numpy().astype(np.float64)
    for sh in shapes:
        n = int(np.prod(sh[1:]))
        out.append(x[:, o:o + n].reshape(sh))
        o += n
    return out


@pytest.mark.parametrize("name", ["learn_A_full", "learn_A_window", "learn_A_cat", "learn_A_long"])
def test_obs_model_matches_reference_fixture(name):
    from pymdp_b200 import ffi
    d = load_golden(name)
    S, O, T, Bn = d["S"].tolist(), d["O"].tolist(), int(d["T"]), int(d["Bn"])
    deps = _deps(d)
    A, pA, obs, qs = unpack(d, "A"), unpack(d, "pA"), unpack(d, "obs"), unpack(d, "qs")
    lay = ffi.EfeLayout(S, O, [1] * len(S), 1, deps, [[f] for f in range(len(S))])
    pA_t, A_t = flat(pA, Bn), flat(A, Bn)
    pA0, A0 = pA_t.clone(), A_t.clone()
    cat = bool(d["categorical"])
    if cat:
        o = cuda(np.concatenate([x.reshape(Bn, T, -1) for x in obs], axis=-1))
    else:
        o = cuda(np.stack(obs, axis=-1), torch.int32)
    q = cuda(np.concatenate(qs, axis=-1))
    mask = sum(1 << m for m in range(len(O)) if not d["none_mask"][m])
    lay.learn_A(pA_t, A_t, o, q, cuda(d["lr"]), Bn, T, modality_mask=mask, categorical=cat)
    torch.cuda.synchronize()
    shapes = [a.shape for a in A]
    got_p, got_e = split(pA_t, shapes), split(A_t, shapes)
    old_p, old_e = split(pA0, shapes), split(A0, shapes)
    for m in range(len(O)):
        if d["none_mask"][m]:
            np.testing.assert_array_equal(got_p[m], old_p[m])
            np.testing.assert_array_equal(got_e[m], old_e[m])
            continue
        np.testing.assert_allclose(got_p[m], d[f"qA{m}"], rtol=P_RTOL, atol=0)
        np.testing.assert_allclose(got_e[m], d[f"EA{m}"], rtol=E_RTOL, atol=E_ATOL)


@pytest.mark.parametrize("name", ["learn_B_online", "learn_B_window", "learn_B_long"])
def test_transition_model_matches_reference_fixture(name):
    from pymdp_b200 import ffi
    d = load_golden(name)
    S, U, T, Bn = d["S"].tolist(), d["U"].tolist(), int(d["T"]), int(d["Bn"])
    deps = _deps(d)
    B, pB, qs = unpack(d, "B"), unpack(d, "pB"), unpack(d, "qs")
    lay = ffi.EfeLayout(S, [2], U, 1, [[0]], deps)
    pB_t, B_t = flat(pB, Bn), flat(B, Bn)
    work = torch.zeros(1, dtype=torch.int32, device="cuda")
    lay.learn_B(pB_t, B_t, cuda(np.concatenate(qs, axis=-1)), cuda(d["actions"], torch.int32), cuda(d["lr"]), work,
                Bn, T, factor_mask=int(d["factor_mask"]))
    torch.cuda.synchronize()
    shapes = [b.shape for b in B]
    got_p, got_e = split(pB_t, shapes), split(B_t, shapes)
    for f in range(len(S)):
        np.testing.assert_allclose(got_p[f], d[f"qB{f}"], rtol=P_RTOL, atol=0)
        np.testing.assert_allclose(got_e[f], d[f"EB{f}"], rtol=E_RTOL, atol=E_ATOL)


def test_transition_model_without_valid_transition_writes_nothing():
    """No agent with a valid transition: pB and B stay bit-identical, B is
    not renormalised (pymdp/agent.py:495-500, :603-604)."""
    from pymdp_b200 import ffi
    d = load_golden("learn_B_online")
    S, U, T, Bn = d["S"].tolist(), d["U"].tolist(), int(d["T"]), int(d["Bn"])
    B, pB, qs = unpack(d, "B"), unpack(d, "pB"), unpack(d, "qs")
    lay = ffi.EfeLayout(S, [2], U, 1, [[0]], _deps(d))
    pB_t, B_t = flat(pB, Bn), flat([x * 1.5 for x in B], Bn)
    pB0, B0 = pB_t.clone(), B_t.clone()
    work = torch.zeros(1, dtype=torch.int32, device="cuda")
    act = np.full_like(d["actions"], -1)
    act[:, :, 1] = 0  # one factor valid is not enough: every factor's action must be >= 0
    lay.learn_B(pB_t, B_t, cuda(np.concatenate(qs, axis=-1)), cuda(act, torch.int32), cuda(d["lr"]), work, Bn, T)
    torch.cuda.synchronize()
    assert torch.equal(pB_t, pB0) and torch.equal(B_t, B0)
    # a single valid transition anywhere renormalises every agent
    act[0, 0, :] = 0
    lay.learn_B(pB_t, B_t, cuda(np.concatenate(qs, axis=-1)), cuda(act, torch.int32), cuda(d["lr"]), work, Bn, T)
    torch.cuda.synchronize()
    got = split(B_t, [b.shape for b in B])
    for f in range(len(S)):
        np.testing.assert_allclose(got[f][1], ol.dirichlet_expected_value(pB[f][1]), rtol=E_RTOL, atol=E_ATOL)


@pytest.mark.parametrize("precision,efe_algorithm", [("fp32", "dense"), ("tf32x3", "dense"), ("fp32", "factored")])
def test_agent_online_learning_loop_matches_oracle(precision, efe_algorithm):
    """Agent.infer_parameters (pymdp/agent.py:416-620) in a closed loop:
    infer_states -> infer_policies -> sample_action -> infer_parameters, three
    steps; A, B, pA, pB and every step's G follow the FP64 oracle fed with the
    same beliefs. The tensor-core precision checks that learning invalidates
    the packed operand images."""
    from pymdp_b200 import Agent
    S, O, U, T = [4, 3], [5, 3], [3, 2], 2
    A_deps, B_deps = [[0, 1], [1]], [[0], [1, 0]]
    rng = np.random.default_rng(11)
    batch = 3

    def dirc(shape, alpha=0.7):
        g = rng.gamma(alpha, size=shape) + 1e-30
        return (g / g.sum(1, keepdims=True)).astype(np.float32)

    A = [dirc((batch, O[m]) + tuple(S[x] for x in A_deps[m])) for m in range(len(O))]
    B = [dirc((batch, S[f]) + tuple(S[x] for x in B_deps[f]) + (U[f],)) for f in range(len(S))]
    C = [rng.normal(size=(batch, o)).astype(np.float32) for o in O]
    pA = [rng.uniform(0.2, 2.0, size=a.shape).astype(np.float32) for a in A]
    pB = [rng.uniform(0.2, 2.0, size=b.shape).astype(np.float32) for b in B]
    agent = Agent(A, B, C=C, A_dependencies=A_deps, B_dependencies=B_deps, policy_len=T, gamma=16.0,
                  batch_size=batch, pA=pA, pB=pB, learn_A=True, learn_B=True, precision=precision,
                  efe_algorithm=efe_algorithm)
    ref = [[np.asarray(x, np.float64) for x in y] for y in (pA, A, pB, B)]
    pol = oefe.construct_policies(S, U, T)
    lrA = np.array([3.0, 1.0, 0.5], np.float32)
    qs_prev, act_prev = None, None
    for step in range(3):
        obs = [rng.integers(0, o, size=batch) for o in O]
        prior = [torch.full((batch, s), 1.0 / s, device="cuda") for s in S]
        qs = agent.infer_states([cuda(o, torch.int32) for o in obs], prior)
        q_pi, G = agent.infer_policies(qs)
        qs_np = [q.cpu().numpy().astype(np.float64) for q in qs]
        for b in range(batch):
            G_ref = oefe.neg_efe_all_policies(pol, [q[b, 0] for q in qs_np], [a[b] for a in ref[1]],
                                              [x[b] for x in ref[3]], [c[b] for c in C], A_deps, B_deps)
            np.testing.assert_allclose(G[b].cpu().numpy(), G_ref, rtol=2e-5, atol=2e-5 * max(1, np.abs(G_ref).max()))
        act = agent.sample_action(q_pi)
        beliefs_B = None if qs_prev is None else [torch.cat([p, q], dim=1) for p, q in zip(qs_prev, qs)]
        agent.infer_parameters(qs, [cuda(o, torch.int32).unsqueeze(1) for o in obs],
                               act_prev if act_prev is not None else torch.full_like(act, -1),
                               beliefs_B=beliefs_B, lr_pA=lrA, lr_pB=2.0)
        bB = qs_np if qs_prev is None else [np.concatenate([p.cpu().numpy(), q], axis=1).astype(np.float64)
                                            for p, q in zip(qs_prev, qs_np)]
        ref = list(ol.infer_parameters(
            ref[0], ref[1], ref[2], ref[3], qs_np, [o[:, None] for o in obs],
            None if act_prev is None else act_prev.cpu().numpy(), A_deps, B_deps, O, U,
            beliefs_B=None if qs_prev is None else bB, lr_pA=lrA.astype(np.float64), lr_pB=2.0))
        for got, want in zip((agent.pA, agent.A, agent.pB, agent.B), ref):
            for g, w in zip(got, want):
                np.testing.assert_allclose(g.cpu().numpy(), w, rtol=1e-5, atol=1e-7)
        qs_prev, act_prev = qs, act


def test_learning_at_benchmark_size_conserves_mass():
    """256 agents of the benchmark model (S = [32, 16, 8], O = [16, 16, 8, 8, 4],
    every modality on every factor, U = [4, 4, 1]): one online step adds
    exactly lr to each modality's counts and touches only the observed row;
    every A and B column sums to 1."""
    from pymdp_b200 import ffi
    S, O, U = [32, 16, 8], [16, 16, 8, 8, 4], [4, 4, 1]
    Bn = 256
    lay = ffi.EfeLayout(S, O, U, 1, [[0, 1, 2]] * 5, [[0], [1], [2]])
    g = torch.Generator(device="cuda").manual_seed(5)
    nA, nB = int(lay.A_offsets[-1]), int(lay.B_offsets[-1])
    pA = torch.rand((Bn, nA), device="cuda", generator=g) * 2 + 0.1
    pB = torch.rand((Bn, nB), device="cuda", generator=g) * 2 + 0.1
    A, Bm = torch.empty_like(pA), torch.empty_like(pB)
    q = torch.cat([torch.softmax(torch.randn((Bn, 2, s), device="cuda", generator=g) * 3, -1) for s in S], -1)
    obs = torch.stack([torch.randint(0, o, (Bn, 1), device="cuda", generator=g) for o in O], -1).to(torch.int32)
    act = torch.stack([torch.randint(0, u, (Bn, 1), device="cuda", generator=g) for u in U], -1).to(torch.int32)
    lr = torch.full((Bn,), 0.75, device="cuda")
    pA0, pB0 = pA.clone(), pB.clone()
    lay.learn_A(pA, A, obs.contiguous(), q[:, :1].contiguous(), lr, Bn, 1)
    lay.learn_B(pB, Bm, q.contiguous(), act.contiguous(), lr, torch.zeros(1, dtype=torch.int32, device="cuda"), Bn, 2)
    torch.cuda.synchronize()
    dA = (pA.double() - pA0.double())
    for m in range(len(O)):
        seg = dA[:, lay.A_offsets[m]:lay.A_offsets[m + 1]].reshape(Bn, O[m], -1)
        np.testing.assert_allclose(seg.sum(dim=(1, 2)).cpu().numpy(), 0.75, rtol=1e-3)
        rows = torch.arange(O[m], device="cuda")[None, :] != obs[:, 0, m].long()[:, None]
        assert (seg.abs().sum(-1)[rows] == 0).all()
        cols = A[:, lay.A_offsets[m]:lay.A_offsets[m + 1]].double().reshape(Bn, O[m], -1).sum(1)
        np.testing.assert_allclose(cols.cpu().numpy(), 1.0, rtol=1e-5)
    dB = (pB.double() - pB0.double())
    for f in range(len(S)):
        seg = dB[:, lay.B_offsets[f]:lay.B_offsets[f + 1]]
        np.testing.assert_allclose(seg.sum(1).cpu().numpy(), 0.75, rtol=1e-3)
        cols = Bm[:, lay.B_offsets[f]:lay.B_offsets[f + 1]].double().reshape(Bn, S[f], -1).sum(1)
        np.testing.assert_allclose(cols.cpu().numpy(), 1.0, rtol=1e-5)


@pytest.mark.parametrize("T", [1, 2, 3, 4])
@pytest.mark.parametrize("categorical", [False, True])
def test_obs_model_float4_path_matches_oracle(T, categorical):
    """Layouts whose columns, offsets and last dependency axis are multiples of
    4 (and 16-byte aligned buffers) take the float4 kernel; a buffer shifted
    by one float takes the scalar kernel. Both match the FP64 oracle."""
    from pymdp_b200 import ffi
    S, O, deps = [3, 8], [5, 7], [[0, 1], [1]]
    Bn = 5
    rng = np.random.default_rng(40 + T)
    lay = ffi.EfeLayout(S, O, [1, 1], 1, deps, [[0], [1]])
    shapes = [(Bn, O[m]) + tuple(S[f] for f in deps[m]) for m in range(len(O))]
    pA = [rng.uniform(0.05, 3.0, size=sh).astype(np.float32) for sh in shapes]
    A = [np.zeros(sh, np.float32) for sh in shapes]
    qs = [rng.dirichlet(np.ones(s), size=(Bn, T)).astype(np.float32) for s in S]
    if categorical:
        obs = [rng.dirichlet(np.ones(o), size=(Bn, T)).astype(np.float32) for o in O]
        o_dev = cuda(np.concatenate(obs, axis=-1))
    else:
        obs = [rng.integers(0, o, size=(Bn, T)) for o in O]
        o_dev = cuda(np.stack(obs, axis=-1), torch.int32)
    lr = rng.uniform(0.5, 2.0, size=Bn).astype(np.float32)
    q_dev = cuda(np.concatenate(qs, axis=-1))
    n = int(lay.A_offsets[-1])
    results = []
    for shift in (0, 1):
        store = torch.zeros(2 * Bn * n + 8, device="cuda")
        pA_t = store[shift:shift + Bn * n].view(Bn, n)
        A_t = store[Bn * n + 4 + shift:Bn * n + 4 + shift + Bn * n].view(Bn, n)
        pA_t.copy_(flat(pA, Bn))
        lay.learn_A(pA_t, A_t, o_dev, q_dev, cuda(lr), Bn, T, categorical=categorical)
        torch.cuda.synchronize()
        results.append((split(pA_t, shapes), split(A_t, shapes)))
    for b in range(Bn):
        qA, EA = ol.update_obs_likelihood_dirichlet([p[b] for p in pA], [a[b] for a in A], [o[b] for o in obs],
                                                    [q[b] for q in qs], deps, O, lr=float(lr[b]),
                                                    categorical_obs=categorical)
        for got_p, got_e in results:
            for m in range(len(O)):
                np.testing.assert_allclose(got_p[m][b], qA[m], rtol=P_RTOL, atol=0)
                np.testing.assert_allclose(got_e[m][b], EA[m], rtol=E_RTOL, atol=E_ATOL)


def test_transition_learning_from_given_joints_matches_reference():
    """b2_update_state_transition_from_joint on the fixture made by the
    reference's own learning.py with pairwise joints (the smoothing
    algorithms' branch of Agent.infer_parameters)."""
    from pymdp_b200 import ffi
    d = load_golden("learn_B_joint")
    Bn, U = int(d["Bn"]), int(d["U"])
    S = d["pB"].shape[1]
    Tm1 = d["joint"].shape[1]
    lay = ffi.EfeLayout([S], [1], [U], 1, [[0]], [[0]])
    pB = torch.as_tensor(d["pB"].reshape(Bn, -1), device="cuda").float().contiguous()
    B = torch.as_tensor(d["B"].reshape(Bn, -1), device="cuda").float().contiguous()
    joint = torch.as_tensor(d["joint"].reshape(Bn, -1), device="cuda").float().contiguous()
    act = torch.as_tensor(d["actions"], device="cuda").to(torch.int32).contiguous()
    lr = torch.as_tensor(d["lr"], device="cuda").float()
    work = torch.zeros(1, dtype=torch.int32, device="cuda")
    lay.learn_B_joint(pB, B, joint, act, lr, work, Bn, Tm1 + 1)
    np.testing.assert_allclose(pB.cpu().numpy().reshape(d["qB"].shape), d["qB"], rtol=2e-6, atol=1e-7)
    np.testing.assert_allclose(B.cpu().numpy().reshape(d["EB"].shape), d["EB"], rtol=2e-6, atol=1e-7)


def test_transition_learning_from_outer_product_joints_equals_the_filtering_form():
    """Joints formed as q_{t+1} (x) q_t[deps] give the filtering form's update
    (b2_update_state_transition_dirichlet) on a multi-factor model with
    multi-parent transitions and one invalid step."""
    from pymdp_b200 import ffi
    rng = np.random.default_rng(41)
    S, U, B_deps, T, Bn = [3, 4, 2], [2, 3, 1], [[0], [1, 0], [2, 1]], 4, 3
    lay = ffi.EfeLayout(S, [1], U, 1, [[0]], B_deps)
    nB = int(lay.B_offsets[-1])
    pB = torch.as_tensor(rng.uniform(0.2, 2.0, size=(Bn, nB)), device="cuda").float()
    B0 = torch.zeros_like(pB)
    qs = [rng.dirichlet(np.ones(s), size=(Bn, T)).astype(np.float32) for s in S]
    act = np.stack([rng.integers(0, u, size=(Bn, T - 1)) for u in U], -1).astype(np.int32)
    act[1, 2, 0] = -1  # an invalid step: masked in both forms
    joints = []
    for f in range(len(S)):
        parents = [qs[d][:, :-1] for d in B_deps[f]]
        j = qs[f][:, 1:]
        for p in parents:
            j = j[..., None] * p.reshape(p.shape[:2] + (1,) * (j.ndim - 2) + (p.shape[-1],))
        joints.append(j.reshape(Bn, -1))
    joint = torch.as_tensor(np.concatenate(joints, 1), device="cuda").contiguous()
    q_seq = torch.as_tensor(np.concatenate(qs, -1), device="cuda").contiguous()
    act_d = torch.as_tensor(act, device="cuda").contiguous()
    lr = torch.full((Bn,), 0.7, device="cuda")
    w1, w2 = torch.zeros(1, dtype=torch.int32, device="cuda"), torch.zeros(1, dtype=torch.int32, device="cuda")
    pB1, B1, pB2, B2 = pB.clone(), B0.clone(), pB.clone(), B0.clone()
    lay.learn_B(pB1, B1, q_seq, act_d, lr, w1, Bn, T)
    lay.learn_B_joint(pB2, B2, joint, act_d, lr, w2, Bn, T)
    np.testing.assert_allclose(pB2.cpu().numpy(), pB1.cpu().numpy(), rtol=2e-6, atol=1e-7)
    np.testing.assert_allclose(B2.cpu().numpy(), B1.cpu().numpy(), rtol=2e-6, atol=1e-7)


def test_agent_learns_B_from_exact_smoothing_joints():
    """The "exact" smoothing branch end to end on the device: filtered beliefs
    -> hmm.smoothing_exact (pymdp/inference.py:595-634) -> pairwise joints ->
    Agent.infer_parameters(joint_beliefs=...) (pymdp/agent.py:530-567), against
    the FP64 oracle applied to the same joints."""
    from pymdp_b200 import Agent, hmm
    rng = np.random.default_rng(17)
    S, U, O, T, Bn = 6, 3, 4, 5, 4
    A = rng.dirichlet(np.ones(O), size=S).T.astype(np.float32)
    B = np.moveaxis(rng.dirichlet(np.ones(S), size=(S, U)), -1, 0).astype(np.float32)
    pB = rng.uniform(0.5, 2.0, size=(S, S, U)).astype(np.float32)
    agent = Agent([A], [B], pB=[pB], learn_B=True, batch_size=Bn)
    filt = torch.as_tensor(rng.dirichlet(np.ones(S), size=(Bn, T)).astype(np.float32), device="cuda")
    acts = rng.integers(0, U, size=(Bn, T - 1)).astype(np.int32)
    acts[2, 1] = -1  # no action taken at that step: the identity transition, and a masked learning step
    B_dev = torch.as_tensor(np.broadcast_to(B, (Bn,) + B.shape).copy(), device="cuda")
    _, joints = hmm.smoothing_exact([filt], [B_dev], torch.as_tensor(acts, device="cuda"))
    agent.infer_parameters(None, None, torch.as_tensor(acts[..., None], device="cuda"), joint_beliefs=joints,
                           lr_pB=0.5)
    jn = joints[0].cpu().numpy().astype(np.float64)
    for b in range(Bn):
        a = acts[b].astype(np.int64)
        jm = jn[b] * (a >= 0)[:, None, None]  # the reference masks invalid transitions
        qb, eb = ol.update_state_transition_from_joint(pB, jm, np.where(a >= 0, a, 0), U, lr=0.5)
        np.testing.assert_allclose(agent.pB[0][b].cpu().numpy(), qb, rtol=2e-6, atol=1e-7)
        np.testing.assert_allclose(agent.B[0][b].cpu().numpy(), eb, rtol=2e-6, atol=1e-7)
