"""b2_neg_efe_noalloc against b2_neg_efe at FP32 precision, through the C-ABI.

b2_neg_efe_noalloc has no counterpart in the reference. It serves callers that
cannot allocate device memory during a call: a host that owns the GPU through
its own arena, a real-time loop that keeps allocator latency out of its step,
a runtime that forbids allocation inside its handlers. Its workspace is one
fixed device array shared by every call, so its contract is to give the same G
as b2_neg_efe (the EFE tests' tolerance: rtol 1e-5, atol 1e-5) on consecutive
calls that reuse that array. This file is collected last so that a run which
stops at the first failure has already run every other test."""

import numpy as np
import pytest
import torch

from oracle import efe as oefe
from pymdp_b200 import _lib
from pymdp_b200.ffi import EfeLayout

G_RTOL, G_ATOL = 1e-5, 1e-5


def _dirichlet(rng, shape, alpha=0.5):
    g = rng.gamma(alpha, size=shape) + 1e-30
    return (g / g.sum(1, keepdims=True)).astype(np.float32)


def _flat_model(seed, S, O, U, T, A_deps, B_deps, batch):
    """Random model as the flat per-agent buffers of the C-ABI (host arrays)."""
    rng = np.random.default_rng(seed)
    A = [_dirichlet(rng, (batch, O[m]) + tuple(S[d] for d in A_deps[m])) for m in range(len(O))]
    B = [_dirichlet(rng, (batch, S[f]) + tuple(S[d] for d in B_deps[f]) + (U[f],)) for f in range(len(S))]
    C = [rng.normal(size=(batch, T, o)).astype(np.float32) for o in O]
    qs = [_dirichlet(rng, (batch, s), 1.0) for s in S]
    flat = lambda xs: np.concatenate([x.reshape(batch, -1) for x in xs], axis=1)
    lay = EfeLayout(S, O, U, T, A_deps, B_deps)
    pol = oefe.construct_policies(S, U, T).astype(np.int32)
    return lay, dict(pm=pol, qs=flat(qs), A=flat(A), B=flat(B), C=flat(C),
                     I=np.zeros((batch, sum(S)), np.float32), eps=np.full(1, 1e-3, np.float32)), pol.shape[0]


def _args(lay, buf, out, Bn, P, flags, stream):
    """Positional arguments shared by b2_neg_efe and b2_neg_efe_noalloc."""
    c = lay._c
    ptr = lambda t: t.data_ptr()
    n = lambda t: t.numel()
    return (stream, ptr(buf["pm"]), n(buf["pm"]), 0, ptr(buf["qs"]), n(buf["qs"]), ptr(buf["A"]), n(buf["A"]),
            ptr(buf["B"]), n(buf["B"]), ptr(buf["C"]), n(buf["C"]), ptr(buf["I"]), n(buf["I"]), None, 0, None, 0,
            ptr(buf["eps"]), n(buf["eps"]), ptr(out), n(out), Bn, P, lay.T, lay.F, lay.M, c[0], c[1], c[2], c[3],
            c[4], c[5], c[6], c[7], c[8], c[9], len(lay.A_dep_flat), c[10], c[11], len(lay.B_dep_flat), c[12],
            flags)


def _workspace_floats(lay, batch):
    return batch * lay.T * sum(int(np.prod([lay.S[d] for d in deps])) for deps in lay.A_dependencies)


MODELS = [
    dict(seed=11, S=[3, 4, 2], O=[4, 5, 3], U=[2, 3, 2], T=2, A_deps=[[0, 2], [1, 2, 0], [1]],
         B_deps=[[0], [1, 0], [2, 1]], batch=5),
    dict(seed=12, S=[8, 6, 4], O=[6, 5], U=[3, 2, 2], T=2, A_deps=[[0, 1, 2], [2, 0, 1]],
         B_deps=[[0], [1, 0], [2]], batch=64),
]


@pytest.mark.gpu
def test_noalloc_matches_neg_efe_on_consecutive_calls():
    lib = _lib.load()
    flags = _lib.FLAG_USE_UTILITY | _lib.FLAG_USE_STATES_INFO_GAIN
    stream = torch.cuda.current_stream().cuda_stream
    runs = []
    for spec in MODELS:
        spec = dict(spec)
        batch = spec.pop("batch")
        lay, host, P = _flat_model(spec.pop("seed"), **spec, batch=batch)
        buf = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
        ref = torch.empty((batch, P), device="cuda")
        _lib.check(lib.b2_neg_efe(*_args(lay, buf, ref, batch, P, flags, stream)))
        runs.append((lay, buf, batch, P, ref))
    # The larger workspace first, then a smaller one with other values: the
    # second call must not pick up what the first left in the shared array.
    runs.sort(key=lambda r: -_workspace_floats(r[0], r[2]))
    outs = []
    for lay, buf, batch, P, _ in runs:
        out = torch.full((batch, P), float("nan"), device="cuda")
        _lib.check(lib.b2_neg_efe_noalloc(*_args(lay, buf, out, batch, P, flags, stream)))
        outs.append(out)
    torch.cuda.synchronize()
    for (lay, buf, batch, P, ref), out in zip(runs, outs):
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        np.testing.assert_allclose(got, ref.cpu().numpy(), rtol=G_RTOL, atol=G_ATOL)


def _host_call(Bn, flags):
    """A call with valid sizes and dummy non-null pointers whose checks all end
    before any device work (no GPU needed)."""
    lay = EfeLayout([32, 16, 8], [16, 16], [4, 4, 1], 3, [[0, 1, 2], [0, 1, 2]], [[0], [1], [2]])
    P = 4
    S_tot, A_n, B_n = int(lay.qs_offsets[-1]), int(lay.A_offsets[-1]), int(lay.B_offsets[-1])
    C_n, I_n, c = int(lay.C_offsets[-1]), int(lay.I_offsets[-1]), lay._c
    return _lib.load().b2_neg_efe_noalloc(
        None, 1, P * lay.T * lay.F, 0, 1, Bn * S_tot, 1, Bn * A_n, 1, Bn * B_n, 1, Bn * C_n, 1, Bn * I_n, None, 0,
        None, 0, 1, 1, 1, Bn * P, Bn, P, lay.T, lay.F, lay.M, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8],
        c[9], len(lay.A_dep_flat), c[10], c[11], len(lay.B_dep_flat), c[12], flags)


def test_noalloc_rejects_workspace_above_the_fixed_scratch():
    # 2 modalities x 4096 columns x T=3 x 4 bytes = 96 KiB per agent: 171
    # agents need more than the 16 MiB array.
    rc = _host_call(171, _lib.FLAG_USE_UTILITY)
    assert rc == _lib.B2_ERR_UNSUPPORTED
    msg = _lib.last_error()
    assert "efe_noalloc" in msg and str(_lib.NOALLOC_SCRATCH_BYTES) in msg


def test_noalloc_rejects_tensor_core_precision():
    rc = _host_call(1, _lib.FLAG_USE_UTILITY | (_lib.PRECISIONS["bf16"] << _lib.PRECISION_SHIFT))
    assert rc == _lib.B2_ERR_UNSUPPORTED
    assert "B2_PRECISION_FP32" in _lib.last_error()


def test_noalloc_rejects_the_flag_gated_terms():
    for flag in (_lib.FLAG_USE_PARAM_INFO_GAIN, _lib.FLAG_USE_INDUCTIVE):
        rc = _host_call(1, _lib.FLAG_USE_UTILITY | flag)
        assert rc == _lib.B2_ERR_UNSUPPORTED
        assert "utility and state-information-gain" in _lib.last_error()


def test_noalloc_unknown_precision_is_an_invalid_argument():
    rc = _host_call(1, _lib.FLAG_USE_UTILITY | (3 << _lib.PRECISION_SHIFT))
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT
    assert "unknown precision selector" in _lib.last_error()


@pytest.mark.gpu
def test_noalloc_at_the_size_limit_matches_neg_efe():
    """170 agents of two K = 4096 modalities at T = 3 fill 15.9 of the 16 MiB:
    the whole fixed array is addressable and the result equals b2_neg_efe's."""
    lib = _lib.load()
    flags = _lib.FLAG_USE_UTILITY | _lib.FLAG_USE_STATES_INFO_GAIN
    stream = torch.cuda.current_stream().cuda_stream
    S, O, U, T = [32, 16, 8], [16, 16], [2, 1, 1], 3
    batch = 170
    lay, host, P = _flat_model(13, S, O, U, T, [[0, 1, 2], [0, 1, 2]], [[0], [1], [2]], batch)
    assert _workspace_floats(lay, batch) * 4 <= _lib.NOALLOC_SCRATCH_BYTES < _workspace_floats(lay, 171) * 4
    buf = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
    ref = torch.empty((batch, P), device="cuda")
    _lib.check(lib.b2_neg_efe(*_args(lay, buf, ref, batch, P, flags, stream)))
    for _ in range(2):
        out = torch.full((batch, P), float("nan"), device="cuda")
        _lib.check(lib.b2_neg_efe_noalloc(*_args(lay, buf, out, batch, P, flags, stream)))
        np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=G_RTOL, atol=G_ATOL)
