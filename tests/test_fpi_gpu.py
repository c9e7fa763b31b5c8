"""FPI parity on the GPU: the sm_100a kernels (through the C-ABI) against the
golden vectors made by the reference's own code and against the FP64 oracle.

Tolerance (FP32 path vs FP64 reference): rtol 1e-5, atol 1e-7 per posterior
entry; size-independent properties (normalisation) at full benchmark size;
out-of-range observations as the reference's all-zero one-hot."""

import numpy as np
import pytest
import torch

from conftest import deps_from, load_golden, unpack
from oracle import fpi as ofpi

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-5, 1e-7
FPI = ["fpi_plain", "fpi_single_factor", "fpi_rank123", "fpi_rank4", "fpi_orphan_factor", "fpi_cfg2",
       "fpi_large"]


def cuda(x, dtype=torch.float32):
    return torch.as_tensor(np.asarray(x), device="cuda").to(dtype)


@pytest.mark.parametrize("name", FPI)
def test_fpi_ffi_ll_form_matches_reference(name):
    from pymdp_b200 import ffi
    d = load_golden(name)
    deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    ll = [cuda(l) for l in unpack(d, "ll")]
    lp = [cuda(ofpi.log_stable(p)) for p in unpack(d, "prior")]
    qs = ffi.fpi_ffi(ll, lp, deps, int(d["num_iter"]))
    for f, q_ref in enumerate(unpack(d, "qs")):
        np.testing.assert_allclose(qs[f].cpu().numpy(), q_ref, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("name", FPI)
def test_fpi_fused_obs_form_matches_reference(name):
    from pymdp_b200 import ffi
    d = load_golden(name)
    deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    qs = ffi.fpi_obs([cuda(a) for a in unpack(d, "A")], cuda(d["obs"], torch.int32),
                     [cuda(p) for p in unpack(d, "prior")], deps, int(d["num_iter"]))
    for f, q_ref in enumerate(unpack(d, "qs")):
        np.testing.assert_allclose(qs[f].cpu().numpy(), q_ref, rtol=RTOL, atol=ATOL)


def random_model(rng, S, O, deps, batch, alpha=0.5, shared=False):
    A = []
    for m, o in enumerate(O):
        shape = (o,) + tuple(S[d] for d in deps[m])
        n = 1 if shared else batch
        g = rng.gamma(alpha, size=(n,) + shape) + 1e-30
        a = (g / g.sum(1, keepdims=True)).astype(np.float32)
        A.append(a[0] if shared else a)
    prior = []
    for s in S:
        g = rng.gamma(1.0, size=(batch, s)) + 1e-30
        prior.append((g / g.sum(1, keepdims=True)).astype(np.float32))
    obs = rng.integers(0, np.array(O), size=(batch, len(O))).astype(np.int32)
    return A, prior, obs


SHAPES = [
    ([1, 5], [3, 2], [[0, 1], [1]]),                 # a single-state factor
    ([33, 2], [4, 7], [[0], [1, 0]]),                # S > 32: several outputs per lane
    ([5, 4, 3, 2, 3], [3, 4], [[0, 1, 2, 3, 4], [4, 2]]),  # rank 5, permuted
    ([2, 2, 2, 2, 2, 2, 2, 2], [3], [[7, 6, 5, 4, 3, 2, 1, 0]]),  # rank 8 (ABI cap)
    ([16, 16, 16, 16], [32] * 6, [[0, 1], [2, 3], [1, 3], [0, 2], [3, 0], [2, 1]]),
    ([3] * 16, [2] * 32, [[m % 16, (m + 5) % 16] for m in range(32)]),  # F = 16, M = 32 limits
    # two-step rank-3 kernel: the agent-step model (float4 loads), S = 64 (two states a lane)
    # with rank-1/2 groups beside, and two rank-3 groups with K % 4 != 0 (scalar loads)
    ([32, 16, 8], [16, 16, 8, 8, 4], [[0, 1, 2]] * 5),
    ([64, 5, 3], [3, 4, 5], [[0, 1, 2], [2, 0], [1]]),
    ([7, 5, 3, 6], [3, 2, 4, 5], [[0, 1, 2], [1, 3], [3, 2, 0], [2]]),
    # more X / Y entries than two per thread (64 x 40 = 2560 at 512 threads): the per-sweep addressing path
    ([64, 32, 8], [3, 2], [[0, 1, 2], [1, 2]]),
]


@pytest.mark.parametrize("shape", SHAPES, ids=[f"S{len(s[0])}M{len(s[1])}-{i}" for i, s in enumerate(SHAPES)])
@pytest.mark.parametrize("shared", [False, True])
def test_fpi_random_shapes_match_oracle(shape, shared):
    from pymdp_b200 import ffi
    S, O, deps = shape
    rng = np.random.default_rng(len(S) * 100 + len(O) + shared)
    batch = 5
    A, prior, obs = random_model(rng, S, O, deps, batch, shared=shared)
    qs = ffi.fpi_obs([cuda(a) for a in A], cuda(obs, torch.int32), [cuda(p) for p in prior], deps, 16)
    A64 = [a.astype(np.float64) for a in A]
    ref = ofpi.run_fpi_batch(A64, obs, [p.astype(np.float64) for p in prior], deps, 16)
    for f in range(len(S)):
        np.testing.assert_allclose(qs[f].cpu().numpy(), ref[f], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("num_iter", [1, 2, 7])
def test_fpi_iteration_counts(num_iter):
    from pymdp_b200 import ffi
    S, O, deps = [4, 3, 5], [6, 2], [[0, 2], [1, 2, 0]]
    rng = np.random.default_rng(num_iter)
    A, prior, obs = random_model(rng, S, O, deps, 3)
    qs = ffi.fpi_obs([cuda(a) for a in A], cuda(obs, torch.int32), [cuda(p) for p in prior], deps, num_iter)
    ref = ofpi.run_fpi_batch([a.astype(np.float64) for a in A], obs, [p.astype(np.float64) for p in prior],
                             deps, num_iter)
    for f in range(3):
        np.testing.assert_allclose(qs[f].cpu().numpy(), ref[f], rtol=RTOL, atol=ATOL)


def test_fpi_full_size_cfg2_properties_and_sample_parity():
    """4096 agents, 4 x 16 states, 6 x 32 obs, rank-2 deps, per-agent A."""
    from pymdp_b200 import ffi
    rng = np.random.default_rng(2)
    S, O = [16] * 4, [32] * 6
    deps = [sorted(rng.choice(4, 2, replace=False).tolist()) for _ in range(6)]
    batch = 4096
    A, prior, obs = random_model(rng, S, O, deps, batch)
    qs = ffi.fpi_obs([cuda(a) for a in A], cuda(obs, torch.int32), [cuda(p) for p in prior], deps, 16)
    q = torch.cat(qs, dim=1).cpu().numpy()
    assert np.isfinite(q).all()
    for f in range(4):
        np.testing.assert_allclose(q[:, 16 * f:16 * (f + 1)].sum(1), 1.0, rtol=0, atol=2e-6)
    idx = rng.choice(batch, 12, replace=False)
    ref = ofpi.run_fpi_batch([a[idx].astype(np.float64) for a in A], obs[idx],
                             [p[idx].astype(np.float64) for p in prior], deps, 16)
    for f in range(4):
        np.testing.assert_allclose(qs[f].cpu().numpy()[idx], ref[f], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("name", ["fpi_bad_obs", "fpi_bad_obs_single"])
def test_fpi_out_of_range_observation_matches_reference(name):
    """An observation outside [0, O_m) is the reference's all-zero one-hot:
    that modality adds nothing (fixture from the reference's own
    run_factorized_fpi, tests/golden/make_golden_edges.py). The fast rank-2
    kernel and the general kernel both see such agents."""
    from pymdp_b200 import ffi
    d = load_golden(name)
    deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    qs = ffi.fpi_obs([cuda(a) for a in unpack(d, "A")], cuda(d["obs"], torch.int32),
                     [cuda(p) for p in unpack(d, "prior")], deps, int(d["num_iter"]))
    for f, q_ref in enumerate(unpack(d, "qs")):
        np.testing.assert_allclose(qs[f].cpu().numpy(), q_ref, rtol=RTOL, atol=ATOL)


def test_fpi_out_of_range_observation_on_the_rank2_fast_path():
    """The benchmark FPI model (the fast rank-2 kernel, 16-byte slice loads):
    agents with out-of-range observations equal the oracle with zero one-hots."""
    from pymdp_b200 import ffi
    rng = np.random.default_rng(12)
    S, O = [16] * 4, [32] * 6
    deps = [sorted(rng.choice(4, 2, replace=False).tolist()) for _ in O]
    A, prior, obs = random_model(rng, S, O, deps, 6)
    obs[1, 0], obs[2, 3], obs[3, :] = -1, 32, 1000
    obs[4, 1], obs[4, 2] = -7, 40
    qs = ffi.fpi_obs([cuda(a) for a in A], cuda(obs, torch.int32), [cuda(p) for p in prior], deps, 16)
    ref = ofpi.run_fpi_batch([a.astype(np.float64) for a in A], obs, [p.astype(np.float64) for p in prior], deps, 16)
    for f in range(4):
        np.testing.assert_allclose(qs[f].cpu().numpy(), ref[f], rtol=RTOL, atol=ATOL)
    # all observations out of range: the posterior is the FPI of the prior alone
    np.testing.assert_allclose(qs[0].cpu().numpy()[3], prior[0][3], rtol=1e-5, atol=1e-7)


def test_fpi_out_of_range_observation_on_the_rank3_two_step_path():
    """The agent-step model (the two-step rank-3 kernel): out-of-range
    observations add nothing, as the oracle's zero one-hots."""
    from pymdp_b200 import ffi
    rng = np.random.default_rng(13)
    S, O, deps = [32, 16, 8], [16, 16, 8, 8, 4], [[0, 1, 2]] * 5
    A, prior, obs = random_model(rng, S, O, deps, 4)
    obs[0, 1], obs[1, :], obs[2, 4] = -1, 99, 4
    qs = ffi.fpi_obs([cuda(a) for a in A], cuda(obs, torch.int32), [cuda(p) for p in prior], deps, 16)
    ref = ofpi.run_fpi_batch([a.astype(np.float64) for a in A], obs, [p.astype(np.float64) for p in prior], deps, 16)
    for f in range(3):
        np.testing.assert_allclose(qs[f].cpu().numpy(), ref[f], rtol=RTOL, atol=ATOL)


def test_fpi_empty_batch_and_errors():
    from pymdp_b200 import ffi
    from pymdp_b200._lib import InvalidArgumentError
    S, O, deps = [4, 3], [5, 2], [[0, 1], [1]]
    A, prior, obs = random_model(np.random.default_rng(1), S, O, deps, 1)
    empty = ffi.fpi_obs([cuda(a[:0]) for a in A], cuda(obs[:0], torch.int32), [cuda(p[:0]) for p in prior],
                        deps, 4)
    assert all(q.shape[0] == 0 for q in empty)
    with pytest.raises(ValueError):
        ffi.fpi_obs([cuda(a) for a in A], cuda(obs, torch.int32), [cuda(p) for p in prior], [[0, 0], [1]], 4)
    with pytest.raises(InvalidArgumentError):
        ffi.fpi_obs_flat(cuda(np.zeros(3)), 3, [0, 1, 2], [1, 1], cuda(obs, torch.int32), cuda(np.zeros((1, 7))),
                         S, deps, 4)
