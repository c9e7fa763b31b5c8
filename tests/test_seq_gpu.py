"""Sequence inference on the GPU (b2_sequence_infer through pymdp_b200.seq):
run_mmp / run_vmp against the golden fixtures made by the reference's own
pymdp/algos.py (tests/golden/make_golden_seq.py) and against the FP64 oracle
on batches of random windows. FP64 inside, FP32 out: rtol 1e-5, atol 1e-7."""

import numpy as np
import pytest
import torch

from conftest import load_golden, unpack
from oracle import mmp

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-5, 1e-7


def _deps(d, key):
    out, i = [], 0
    for n in d[key + "_len"]:
        out.append(d[key + "_flat"][i:i + n].tolist())
        i += n
    return out


def cuda(x, dtype=torch.float32):
    return torch.as_tensor(np.asarray(x), device="cuda").to(dtype)


@pytest.mark.parametrize("name", ["seq_mmp", "seq_mmp_index", "seq_vmp", "seq_vmp_index", "seq_mmp_bench",
                                  "seq_vmp_bench", "seq_mmp_rank3", "seq_vmp_t1"])
def test_sequence_inference_matches_reference(name):
    from pymdp_b200 import seq
    d = load_golden(name)
    fn = seq.run_mmp if str(d["kind"]) == "mmp" else seq.run_vmp
    distr = bool(d["distr"])
    obs = [cuda(o[None]) if distr else cuda(o[None], torch.int32) for o in unpack(d, "obs")]
    qs = fn([cuda(a) for a in unpack(d, "A")], [cuda(b[None]) for b in unpack(d, "B")], obs,
            [cuda(p[None]) for p in unpack(d, "prior")], _deps(d, "A_deps"), _deps(d, "B_deps"),
            num_iter=int(d["num_iter"]), tau=float(d["tau"]), distr_obs=distr)
    for got, want in zip(qs, unpack(d, "qs")):
        np.testing.assert_allclose(got[0].cpu().numpy(), want, rtol=RTOL, atol=ATOL)


def _cols(rng, shape, alpha=0.7):
    g = np.maximum(rng.gamma(alpha, size=shape), 1e-30)
    return (g / g.sum(0, keepdims=True)).astype(np.float32)


@pytest.mark.parametrize("kind", ["mmp", "vmp"])
@pytest.mark.parametrize("distr", [False, True])
@pytest.mark.parametrize("case", [
    dict(S=[4, 3], O=[5, 2], A_deps=[[0, 1], [1]], B_deps=[[0], [1, 0]], T=6, num_iter=10, tau=0.5),
    dict(S=[3, 2, 4], O=[3, 4, 2], A_deps=[[2, 0], [1], [0, 1, 2]], B_deps=[[0, 2], [1], [2]], T=3, num_iter=4,
         tau=1.0),
    dict(S=[5], O=[3], A_deps=[[0]], B_deps=[[0]], T=1, num_iter=3, tau=0.25),
    # transition sequences too large to stage in shared memory (read from global memory): single-parent and
    # multi-parent
    dict(S=[100], O=[6], A_deps=[[0]], B_deps=[[0]], T=8, num_iter=3, tau=0.5),
    dict(S=[40, 30], O=[7, 5], A_deps=[[0, 1], [1]], B_deps=[[0, 1], [1]], T=5, num_iter=3, tau=0.5),
])
def test_batched_sequence_inference_matches_oracle(case, kind, distr):
    from pymdp_b200 import seq
    rng = np.random.default_rng(len(case["S"]) * 10 + case["T"])
    S, O, T, batch = case["S"], case["O"], case["T"], 5
    A = [np.stack([_cols(rng, (O[m],) + tuple(S[d] for d in case["A_deps"][m])) for _ in range(batch)])
         for m in range(len(O))]
    B = [np.stack([np.moveaxis(_cols(rng, (S[f], max(T - 1, 0)) + tuple(S[d] for d in case["B_deps"][f]), 0.5), 1, 0)
                   for _ in range(batch)]) for f in range(len(S))]
    prior = [np.stack([_cols(rng, (s,), 1.0) for _ in range(batch)]) for s in S]
    if distr:
        obs = [np.stack([np.moveaxis(_cols(rng, (O[m], T), 0.5), 1, 0) for _ in range(batch)]) for m in range(len(O))]
    else:
        obs = [rng.integers(0, O[m], size=(batch, T)) for m in range(len(O))]
    fn = seq.run_mmp if kind == "mmp" else seq.run_vmp
    qs = fn([cuda(a) for a in A], [cuda(b) for b in B],
            [cuda(o) if distr else cuda(o, torch.int32) for o in obs], [cuda(p) for p in prior],
            case["A_deps"], case["B_deps"], num_iter=case["num_iter"], tau=case["tau"], distr_obs=distr)
    for b in range(batch):
        ref = mmp.run_sequence(kind, [a[b] for a in A], [x[b] for x in B], [o[b] for o in obs], [p[b] for p in prior],
                               case["A_deps"], case["B_deps"], num_iter=case["num_iter"], tau=case["tau"],
                               distr_obs=distr)
        for f in range(len(S)):
            np.testing.assert_allclose(qs[f][b].cpu().numpy(), ref[f], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("kind", ["mmp", "vmp"])
def test_prepared_plan_reruns_equal_the_list_call(kind):
    """seq.prepare packs the inputs once; every run() of the plan gives the
    list-taking call's posteriors bitwise (the same kernel on the same
    values)."""
    from pymdp_b200 import seq
    rng = np.random.default_rng(29)
    S, O, T, batch = [4, 3], [5, 2], 5, 7
    A_deps, B_deps = [[0, 1], [1]], [[0], [1, 0]]
    A = [cuda(np.stack([_cols(rng, (O[m],) + tuple(S[d] for d in A_deps[m])) for _ in range(batch)]))
         for m in range(len(O))]
    B = [cuda(np.stack([np.moveaxis(_cols(rng, (S[f], T - 1) + tuple(S[d] for d in B_deps[f]), 0.5), 1, 0)
                        for _ in range(batch)])) for f in range(len(S))]
    prior = [cuda(np.stack([_cols(rng, (s,), 1.0) for _ in range(batch)])) for s in S]
    obs = [cuda(rng.integers(0, O[m], size=(batch, T)), torch.int32) for m in range(len(O))]
    fn = seq.run_mmp if kind == "mmp" else seq.run_vmp
    want = fn(A, B, obs, prior, A_deps, B_deps, num_iter=6, tau=0.5, distr_obs=False)
    plan = seq.prepare(kind == "vmp", A, B, obs, prior, A_deps, B_deps, num_iter=6, tau=0.5, distr_obs=False)
    for _ in range(3):
        got = plan.run()
        torch.cuda.synchronize()
        for f in range(len(S)):
            assert torch.equal(got[f], want[f])
