"""C-ABI checks that need no GPU: the library loads, exports every symbol
declared in include/pymdp_b200.h, and its host-side validation rejects the
inputs the reference's validators reject (pymdp/ffi/fpi/fpi_entry.h:24-82,
pymdp/ffi/neg_efe/neg_efe_layout.h:269-363) before touching the device."""

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from pymdp_b200 import _lib

HEADER = os.path.join(ROOT, "include", "pymdp_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(b2_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 9
    for s in syms:
        assert hasattr(lib, s), s
    assert lib.b2_abi_version() >= 1
    assert lib.b2_capabilities() & (1 << 2)
    assert _lib.launch_count() >= 0


def _fpi(S, ll_offsets, lp_offsets, dep_flat, dep_offs, num_iter, ll_count, lp_count, q_count):
    lib = _lib.load()
    i64 = _lib.i64
    return lib.b2_fpi(None, 1, ll_count, 1, lp_count, 1, q_count, i64(S), len(S), i64(ll_offsets),
                      len(ll_offsets), i64(lp_offsets), len(lp_offsets), i64(dep_flat), len(dep_flat),
                      i64(dep_offs), len(dep_offs), num_iter)


GOOD = dict(S=[3, 2], ll_offsets=[0, 6, 12], lp_offsets=[0, 3, 5], dep_flat=[0, 1, 0, 1], dep_offs=[0, 2, 4],
            num_iter=16, ll_count=12, lp_count=5, q_count=5)


@pytest.mark.parametrize("change,msg", [
    (dict(num_iter=0), "num_iter = 0, must be positive"),
    (dict(S=[3, 0]), "S[1] must be positive"),
    (dict(dep_flat=[0, 0, 0, 1]), "duplicate factor"),
    (dict(dep_flat=[0, 2, 0, 1]), "out of range"),
    (dict(lp_offsets=[0, 3]), "lp_offsets size = 2, expected 3"),
    (dict(ll_offsets=[0, 6, 11], ll_count=11), "ll_offsets inconsistent"),
    (dict(lp_count=7), "not divisible by total_S"),
    (dict(ll_count=13), "ll_flat element_count = 13, expected 12"),
    (dict(q_count=10), "q_out element_count = 10, expected 5"),
    (dict(dep_flat=list(range(9)) + [0, 1], dep_offs=[0, 9, 11], S=[2] * 9,
          lp_offsets=list(range(0, 20, 2)), lp_count=18, q_count=18), "rank 9 outside [1, 8]"),
])
def test_fpi_validation_errors(change, msg):
    args = dict(GOOD)
    args.update(change)
    rc = _fpi(**args)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT, (rc, _lib.last_error())
    assert msg in _lib.last_error()
    assert _lib.last_error().startswith("fpi_ffi:")


def test_fpi_limits_are_reported_as_unsupported():
    F = 17
    rc = _fpi(S=[2] * F, ll_offsets=[0, 2], lp_offsets=list(range(0, 2 * F + 1, 2)), dep_flat=[0],
              dep_offs=[0, 1], num_iter=1, ll_count=2, lp_count=2 * F, q_count=2 * F)
    assert rc == _lib.B2_ERR_UNSUPPORTED
    assert "limits" in _lib.last_error()


def _efe_layout_args(S=(3, 2), O=(3, 5), U=(3, 1), T=1, A_deps=((0, 1), (0, 1)), B_deps=((0,), (1,))):
    from pymdp_b200.ffi import EfeLayout
    return EfeLayout(S, O, U, T, A_deps, B_deps)


def _efe_call(lay, Bn=0, P=3, flags=3, counts=None):
    lib = _lib.load()
    c = lay._c
    cnt = dict(pm=P * lay.T * lay.F, qs=Bn * lay.qs_offsets[-1], A=Bn * lay.A_offsets[-1],
               B=Bn * lay.B_offsets[-1], C=Bn * lay.C_offsets[-1], I=Bn * lay.I_offsets[-1], pA=0, pB=0, eps=1,
               out=Bn * P)
    cnt.update(counts or {})
    return lib.b2_neg_efe(None, 1, cnt["pm"], 0, 1, cnt["qs"], 1, cnt["A"], 1, cnt["B"], 1, cnt["C"], 1, cnt["I"],
                          1, cnt["pA"], 1, cnt["pB"], 1, cnt["eps"], 1, cnt["out"], Bn, P, lay.T, lay.F, lay.M,
                          c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[9], len(lay.A_dep_flat), c[10],
                          c[11], len(lay.B_dep_flat), c[12], flags)


def test_efe_valid_empty_batch_is_a_noop():
    assert _efe_call(_efe_layout_args(), Bn=0) == _lib.B2_OK


@pytest.mark.parametrize("counts,msg", [
    (dict(A=5), "A element_count = 5, expected 0"),
    (dict(pm=4), "policy_matrix element_count = 4, expected 6"),
    (dict(eps=3), "inductive_epsilon must have 1 or Bn elements"),
])
def test_efe_count_errors(counts, msg):
    rc = _efe_call(_efe_layout_args(), Bn=0, P=3, counts=counts)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT
    assert msg in _lib.last_error() and _lib.last_error().startswith("efe_ffi:")


def test_efe_layout_errors():
    lay = _efe_layout_args()
    lay.B_offsets[2] += 1
    lay._c[5] = _lib.i64(lay.B_offsets)
    assert _efe_call(lay) == _lib.B2_ERR_INVALID_ARGUMENT
    assert "B_off inconsistent" in _lib.last_error()
    lay = _efe_layout_args()
    lay.A_dep_flat[3] = 3
    lay._c[9] = _lib.i64(lay.A_dep_flat)
    assert _efe_call(lay) == _lib.B2_ERR_INVALID_ARGUMENT
    assert "out of range" in _lib.last_error()


def test_efe_flag_gated_terms_validation():
    """Inductive (bit 2) and parameter information gain (bit 3): the count
    checks of neg_efe_layout.h, before any device work (empty batch)."""
    lay = _efe_layout_args()
    assert _efe_call(lay, flags=3 | 4) == _lib.B2_OK
    assert _efe_call(lay, flags=3 | 8) == _lib.B2_ERR_INVALID_ARGUMENT
    assert "requires at least one of pA, pB" in _lib.last_error()
    assert _efe_call(lay, flags=3 | 8, counts=dict(pA=1)) == _lib.B2_ERR_INVALID_ARGUMENT
    assert "pA element_count = 1, expected 0" in _lib.last_error()
    assert _efe_call(lay, flags=3 | 8, counts=dict(pB=2)) == _lib.B2_ERR_INVALID_ARGUMENT
    assert "pB element_count = 2, expected 0" in _lib.last_error()


def test_construct_policies_matches_oracle_order():
    from oracle.efe import construct_policies as ref
    from pymdp_b200.control import construct_policies
    for S, U, T in [([3, 2], [3, 1], 1), ([32, 16, 8], [4, 4, 1], 3), ([4, 3, 2], [3, 2, 1], 2)]:
        np.testing.assert_array_equal(construct_policies(S, U, T), ref(S, U, T))


def test_package_imports_without_gpu():
    import pymdp_b200
    from pymdp_b200 import Agent, ffi  # noqa: F401
    assert callable(ffi.fpi_ffi) and callable(ffi.neg_efe_all_policies_ffi)
    assert pymdp_b200.Agent is Agent
    assert ffi.is_available()


def test_generate_I_matrix_matches_reference_fixture():
    """pymdp_b200.control.generate_I_matrix against the I the reference's
    generate_I_matrix (pymdp/control.py:965-1019) produced for the stored
    goal vectors H (threshold 0.1, depth 3)."""
    from conftest import load_golden, unpack
    from pymdp_b200.control import generate_I_matrix
    for name in ("efe_ind", "efe_all"):
        d = load_golden(name)
        I = generate_I_matrix(unpack(d, "H"), unpack(d, "B"), 0.1, 3)
        for got, want in zip(I, unpack(d, "I")):
            np.testing.assert_array_equal(got, want)


def test_fit_model_multiaction_map_matches_oracle():
    """Host logic of the fitting likelihood: the policy -> multi-action map
    reproduces ``multiaction_probabilities`` (``pymdp/agent.py:908-937``)."""
    import torch

    from oracle import fitting as ofit
    from pymdp_b200.fitting import FitModel
    for S, U, T in (([8, 4], [4, 1], 2), ([3, 2, 2], [3, 1, 2], 2), ([4], [4], 3)):
        fm = FitModel(S, [3] * len(S), U, policy_len=T, device="cpu")
        rng = np.random.default_rng(1)
        q = rng.dirichlet(np.ones(fm.P))
        got = (torch.as_tensor(q, dtype=torch.float32) @ fm.policy_to_multi).numpy()
        ref = ofit.multiaction_probabilities(q, fm.policies.numpy(), U)
        np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-7)


def test_neg_efe_pack_bytes_host_query():
    """b2_neg_efe_pack_bytes plans the tensor-core operand images on the host:
    positive for the tensor-core precisions, 0 where the SIMT path runs."""
    from pymdp_b200 import ffi
    lay = ffi.EfeLayout([32, 16, 8], [16, 16, 8, 8, 4], [4, 4, 1], 3, [[0, 1, 2]] * 5, [[0], [1], [2]])
    P = 16 ** 3
    n_tf = lay.pack_bytes(4, P, ffi.efe_flags(precision="tf32x3"))
    n_bf = lay.pack_bytes(4, P, ffi.efe_flags(precision="bf16"))
    assert n_tf > n_bf > 0 and n_tf % 4 == 0 and n_bf % 4 == 0
    assert lay.pack_bytes(8, P, ffi.efe_flags(precision="bf16")) == 2 * n_bf
    assert lay.pack_bytes(4, P, ffi.efe_flags(precision="fp32")) == 0
    assert lay.pack_bytes(4, P, ffi.efe_flags(use_inductive=True, precision="bf16")) == 0


def test_sample_action_validation():
    """b2_sample_action rejects bad modes and sizes before touching a GPU."""
    import ctypes
    lib = _lib.load()
    U = (ctypes.c_int64 * 2)(3, 2)
    rc = lib.b2_sample_action(None, 0x1000, 0x1000, U, 0x1000, 4, 6, 1, 2, 2, 0, 0x1000, 0, 0)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and b"sampling_mode" in lib.b2_last_error()
    rc = lib.b2_sample_action(None, 0x1000, 0x1000, U, 0x1000, 4, 6, 1, 2, 0, 3, 0x1000, 0, 0)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and b"action_selection" in lib.b2_last_error()
    big = (ctypes.c_int64 * 2)(3, 4096)
    rc = lib.b2_sample_action(None, 0x1000, 0x1000, big, 0x1000, 4, 6, 1, 2, 1, 0, 0x1000, 0, 0)
    assert rc == _lib.B2_ERR_UNSUPPORTED
    rc = lib.b2_sample_action(None, 0x1000, 0x1000, None, 0x1000, 4, 6, 1, 2, 1, 0, 0x1000, 0, 0)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT


def test_pipelined_step_needs_both_inputs():
    """PipelinedAgentStep alternates two buffer sets: a set's buffers hold the
    inputs of two steps back, so an omitted input is an error, raised before
    any device work."""
    from pymdp_b200.agent import PipelinedAgentStep
    pipe = PipelinedAgentStep.__new__(PipelinedAgentStep)  # no device: the check comes first
    with pytest.raises(ValueError, match="both"):
        pipe.step(None, np.zeros((1, 3), np.float32))
    with pytest.raises(ValueError, match="both"):
        pipe.step(np.zeros((1, 2), np.int32), None)


def _seq(S=(3,), O=(2,), A_deps=((0,),), B_deps=((0,),), T=4, Bn=0, num_iter=4, counts=None, index_obs=True):
    """b2_sequence_infer with host-side arguments only: every case here is
    decided by the validation before any device work (Bn = 0 or an error)."""
    lib = _lib.load()
    i64 = _lib.i64
    size = lambda d: S[d] if 0 <= d < len(S) else 1  # noqa: E731 (out-of-range deps are the library's to reject)
    K = [int(np.prod([size(d) for d in deps])) for deps in A_deps]
    Kb = [int(np.prod([size(d) for d in deps])) for deps in B_deps]
    c = dict(A=sum(o * k for o, k in zip(O, K)), obs=Bn * T * len(O),
             B=Bn * sum((T - 1) * s * kb for s, kb in zip(S, Kb)), prior=Bn * sum(S), qs=Bn * T * sum(S))
    c.update(counts or {})
    adf = [d for deps in A_deps for d in deps]
    ado = list(np.cumsum([0] + [len(d) for d in A_deps]))
    bdf = [d for deps in B_deps for d in deps]
    bdo = list(np.cumsum([0] + [len(d) for d in B_deps]))
    dummy = (ctypes.c_int32 * 1)()  # an observation pointer is required; Bn = 0 never reads it
    obs_idx = ctypes.addressof(dummy) if index_obs else None
    obs_distr = None if index_obs else ctypes.cast(dummy, ctypes.POINTER(ctypes.c_float))
    return lib.b2_sequence_infer(None, 0, None, c["A"], 0, i64(list(O)), len(O), obs_idx, obs_distr, c["obs"], None,
                                 c["B"], None, c["prior"], None, c["qs"], Bn, T, len(S), i64(list(S)), i64(adf),
                                 len(adf), i64(ado), i64(bdf), len(bdf), i64(bdo), num_iter, 0.5)


def test_sequence_empty_batch_is_a_noop():
    assert _seq() == _lib.B2_OK, _lib.last_error()
    assert _seq(S=(4, 3), O=(5, 2), A_deps=((0, 1), (1,)), B_deps=((0,), (1, 0)), T=6) == _lib.B2_OK


@pytest.mark.parametrize("kw,msg", [
    (dict(T=0), "invalid T"),
    (dict(num_iter=-1), "invalid T, num_iter or Bn"),
    (dict(A_deps=((0, 0),), S=(3,)), "duplicate factor in A_dependencies"),
    (dict(A_deps=((1,),)), "A dependency out of range"),
    (dict(B_deps=((2,),)), "B dependency out of range"),
    (dict(counts={"A": 5}), "A element_count mismatch"),
    (dict(Bn=2, counts={"obs": 7}), "observation element_count mismatch"),
    (dict(Bn=2, counts={"B": 1}), "B element_count mismatch"),
    (dict(Bn=2, counts={"qs": 3}), "prior / qs element_count mismatch"),
])
def test_sequence_validation_errors(kw, msg):
    rc = _seq(**kw)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT, (rc, _lib.last_error())
    assert msg in _lib.last_error()
    assert _lib.last_error().startswith("run_mmp:")


def test_sequence_window_beyond_shared_memory_is_unsupported():
    # 8 steps of a 1000-state factor: the FP64 window state alone is about 424 KB
    rc = _seq(S=(1000,), O=(2,), T=8)
    assert rc == _lib.B2_ERR_UNSUPPORTED, (rc, _lib.last_error())
    assert "exceeds 200 KB" in _lib.last_error()


def _expected_state(S=(3, 2), U=(2, 1), B_deps=((0,), (1, 0)), Bn=0, qs_offsets=None, B_offsets=None, counts=None):
    """b2_expected_state with host-side arguments only (Bn = 0 or an error:
    nothing reaches the device)."""
    lib = _lib.load()
    i64 = _lib.i64
    K = [int(np.prod([S[d] if 0 <= d < len(S) else 1 for d in deps])) for deps in B_deps]
    qo = qs_offsets if qs_offsets is not None else list(np.cumsum([0] + list(S)))
    bo = B_offsets if B_offsets is not None else list(np.cumsum([0] + [s * k * u for s, k, u in zip(S, K, U)]))
    c = dict(qs=Bn * sum(S), B=Bn * int(bo[-1]), action=Bn * len(S))
    c.update(counts or {})
    bdf = [d for deps in B_deps for d in deps]
    bdo = list(np.cumsum([0] + [len(d) for d in B_deps]))
    return lib.b2_expected_state(None, None, c["qs"], None, c["B"], None, c["action"], None, Bn, len(S),
                                 i64(list(S)), i64(list(U)), i64(qo), i64(bo), i64(bdf), len(bdf), i64(bdo))


def test_expected_state_empty_batch_is_a_noop():
    assert _expected_state() == _lib.B2_OK, _lib.last_error()


@pytest.mark.parametrize("kw,msg", [
    (dict(S=(3, 0)), "S and U must lie in [1, 4096]"),
    (dict(U=(2, 0)), "S and U must lie in [1, 4096]"),
    (dict(qs_offsets=[0, 3, 4]), "qs_offsets inconsistent with S"),
    (dict(B_offsets=[0, 18, 31]), "B_offsets inconsistent"),
    (dict(B_deps=((0,), (2,))), "B dependency out of range"),
    (dict(Bn=2, counts={"action": 3}), "element counts do not match Bn"),
    (dict(Bn=-1), "negative Bn"),
])
def test_expected_state_validation_errors(kw, msg):
    rc = _expected_state(**kw)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT, (rc, _lib.last_error())
    assert msg in _lib.last_error()
    assert _lib.last_error().startswith("expected_state:")


def _multiaction(U=(3, 2), n_unique=6, marginal=1, Bn=0, P=6, T=1, ptrs=False):
    lib = _lib.load()
    dummy = (ctypes.c_float * 1)()
    q = ctypes.cast(dummy, ctypes.POINTER(ctypes.c_float)) if ptrs else None
    addr = ctypes.addressof(dummy) if ptrs else None
    return lib.b2_multiaction_probabilities(None, q, addr, addr, n_unique, marginal, Bn, P, T, len(U),
                                            _lib.i64(list(U)), q)


def test_multiaction_empty_batch_is_a_noop():
    assert _multiaction() == _lib.B2_OK, _lib.last_error()
    assert _multiaction(marginal=0, n_unique=4) == _lib.B2_OK, _lib.last_error()


@pytest.mark.parametrize("kw,rc,msg", [
    (dict(P=0), "invalid", "invalid sizes"),
    (dict(n_unique=0), "invalid", "invalid sizes"),
    (dict(U=(3, 0)), "invalid", "U must be positive"),
    (dict(n_unique=5), "invalid", "marginal mode writes prod(U) probabilities"),
    (dict(Bn=1), "invalid", "null buffer"),
    # marginal mode keeps one FP64 sum per control in shared memory: 7000 controls are 56 KB
    (dict(U=(7000,), n_unique=7000, Bn=1, ptrs=True), "unsupported", "too many controls"),
])
def test_multiaction_validation_errors(kw, rc, msg):
    want = _lib.B2_ERR_INVALID_ARGUMENT if rc == "invalid" else _lib.B2_ERR_UNSUPPORTED
    got = _multiaction(**kw)
    assert got == want, (got, _lib.last_error())
    assert msg in _lib.last_error()


@pytest.mark.parametrize("Bn,P,rc,msg", [
    (0, 8, "ok", ""),
    (-1, 8, "invalid", "invalid Bn or P"),
    (2, 0, "invalid", "invalid Bn or P"),
    (2, 8, "invalid", "null buffer"),
])
def test_policy_posterior_validation(Bn, P, rc, msg):
    got = _lib.load().b2_policy_posterior(None, None, None, 0, None, 0, None, Bn, P)
    want = _lib.B2_OK if rc == "ok" else _lib.B2_ERR_INVALID_ARGUMENT
    assert got == want, (got, _lib.last_error())
    if msg:
        assert _lib.last_error() == "policy_posterior: " + msg


@pytest.mark.parametrize("Bn,P,T,F,rc,msg", [
    (0, 8, 2, 2, "ok", ""),
    (2, 8, 0, 2, "invalid", "invalid sizes"),
    (2, 8, 2, 0, "invalid", "invalid sizes"),
    (-1, 8, 2, 2, "invalid", "invalid sizes"),
    (2, 8, 2, 2, "invalid", "null buffer"),
])
def test_select_action_validation(Bn, P, T, F, rc, msg):
    got = _lib.load().b2_select_action(None, None, None, None, Bn, P, T, F)
    want = _lib.B2_OK if rc == "ok" else _lib.B2_ERR_INVALID_ARGUMENT
    assert got == want, (got, _lib.last_error())
    if msg:
        assert _lib.last_error() == "select_action: " + msg


def _fpi_obs(S=(3, 2), O=(4, 5), deps=((0, 1), (1,)), A_offsets=None, batch=0, stride=0, num_iter=16, O_len=None):
    """b2_fpi_obs (the fused observation form) with host-side arguments only."""
    lib = _lib.load()
    i64 = _lib.i64
    K = [int(np.prod([S[d] if 0 <= d < len(S) else 1 for d in dd])) for dd in deps]
    ao = A_offsets if A_offsets is not None else list(np.cumsum([0] + [o * k for o, k in zip(O, K)]))
    df = [d for dd in deps for d in dd]
    do = list(np.cumsum([0] + [len(dd) for dd in deps]))
    return lib.b2_fpi_obs(None, None, stride, i64(ao), len(ao), i64(list(O)), len(O) if O_len is None else O_len,
                          None, None, None, batch, i64(list(S)), len(S), i64(df), len(df), i64(do), len(do), num_iter)


def test_fpi_obs_empty_batch_is_a_noop():
    assert _fpi_obs() == _lib.B2_OK, _lib.last_error()


@pytest.mark.parametrize("kw,msg", [
    (dict(O_len=1), "O / A_offsets sizes inconsistent with M = 2"),
    (dict(O=(4, 0)), "must be positive"),
    (dict(A_offsets=[0, 24, 33]), "A_offsets inconsistent with O/deps for modality 1"),
    (dict(A_offsets=[1, 25, 35]), "A_offsets must start at zero"),
    (dict(batch=-1), "negative batch"),
    (dict(stride=10), "A_agent_stride smaller than one agent's A"),
    (dict(batch=2), "null buffer"),
    (dict(num_iter=0), "num_iter = 0, must be positive"),
    (dict(deps=((0, 0), (1,))), "duplicate factor"),
])
def test_fpi_obs_validation_errors(kw, msg):
    rc = _fpi_obs(**kw)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT, (rc, _lib.last_error())
    assert msg in _lib.last_error(), _lib.last_error()
    assert _lib.last_error().startswith("fpi_obs:")


def _fpi_obs_bwd(batch=0, num_iter=16, O=(4, 5)):
    """b2_fpi_obs_bwd (the FPI adjoint) with host-side arguments only."""
    lib = _lib.load()
    i64 = _lib.i64
    S, deps = (3, 2), ((0, 1), (1,))
    K = [6, 2]
    ao = list(np.cumsum([0] + [o * k for o, k in zip(O, K)]))
    return lib.b2_fpi_obs_bwd(None, None, 0, i64(ao), len(ao), i64(list(O)), len(O), None, None, None, None, None,
                              batch, i64(list(S)), len(S), i64([0, 1, 1]), 3, i64([0, 2, 3]), 3, num_iter)


def test_fpi_obs_bwd_validation():
    assert _fpi_obs_bwd() == _lib.B2_OK, _lib.last_error()
    assert _fpi_obs_bwd(batch=-1) == _lib.B2_ERR_INVALID_ARGUMENT
    assert _lib.last_error() == "fpi_obs bwd: negative batch"
    assert _fpi_obs_bwd(batch=3) == _lib.B2_ERR_INVALID_ARGUMENT
    assert _lib.last_error() == "fpi_obs bwd: null buffer"
    assert _fpi_obs_bwd(O=(4, 0)) == _lib.B2_ERR_INVALID_ARGUMENT
    assert "must be positive" in _lib.last_error()
    # the reverse pass keeps every sweep's posterior on chip: 20000 sweeps do not fit
    assert _fpi_obs_bwd(num_iter=20000) == _lib.B2_ERR_UNSUPPORTED, _lib.last_error()
    assert "exceeds shared memory" in _lib.last_error()


def _trans_joint(Bn=0, T=3, S=(3, 2), U=(2, 1), B_deps=((0,), (1, 0)), counts=None, B_offsets=None):
    """b2_update_state_transition_from_joint with host-side arguments only."""
    lib = _lib.load()
    i64 = _lib.i64
    K = [int(np.prod([S[d] if 0 <= d < len(S) else 1 for d in deps])) for deps in B_deps]
    bo = B_offsets if B_offsets is not None else list(np.cumsum([0] + [s * k * u for s, k, u in zip(S, K, U)]))
    c = dict(B=Bn * int(bo[-1]), joint=Bn * sum((T - 1) * s * k for s, k in zip(S, K)), actions=Bn * (T - 1) * len(S))
    c.update(counts or {})
    bdf = [d for deps in B_deps for d in deps]
    bdo = list(np.cumsum([0] + [len(d) for d in B_deps]))
    qo = list(np.cumsum([0] + list(S)))
    return lib.b2_update_state_transition_from_joint(None, None, None, c["B"], None, c["joint"], None, c["actions"],
                                                     None, 0, None, Bn, T, len(S), i64(list(S)), i64(list(U)),
                                                     i64(qo), i64(bo), i64(bdf), len(bdf), i64(bdo), -1)


def test_transition_from_joint_validation():
    op = "update_state_transition_from_joint: "
    assert _trans_joint() == _lib.B2_OK, _lib.last_error()
    assert _trans_joint(Bn=2, T=1) == _lib.B2_OK, _lib.last_error()  # one step: no transition to learn
    cases = [
        (dict(T=0), "invalid sizes"),
        (dict(U=(2, 0)), "num_controls must be positive"),
        (dict(B_offsets=[0, 18, 31]), "B_offsets inconsistent with S, U and dependencies"),
        (dict(Bn=2, counts={"B": 1}), "B_count mismatch"),
        (dict(Bn=2, counts={"joint": 1}), "joint_count mismatch"),
        (dict(Bn=2, counts={"actions": 1}), "actions_count mismatch"),
        (dict(Bn=2), "null buffer"),
    ]
    for kw, msg in cases:
        rc = _trans_joint(**kw)
        assert rc == _lib.B2_ERR_INVALID_ARGUMENT, (kw, rc, _lib.last_error())
        assert _lib.last_error().startswith(op + msg), (kw, _lib.last_error())


def _efe_bwd_call(lay, Bn=0, P=3, flags=3, counts=None):
    """b2_neg_efe_bwd (the neg-EFE adjoint) with host-side arguments only."""
    lib = _lib.load()
    c = lay._c
    cnt = dict(pm=P * lay.T * lay.F, qs=Bn * lay.qs_offsets[-1], A=Bn * lay.A_offsets[-1],
               B=Bn * lay.B_offsets[-1], C=Bn * lay.C_offsets[-1], dG=Bn * P)
    cnt.update(counts or {})
    return lib.b2_neg_efe_bwd(None, None, cnt["pm"], 0, None, cnt["qs"], None, cnt["A"], None, cnt["B"], None,
                              cnt["C"], None, cnt["dG"], None, None, None, None, Bn, P, lay.T, lay.F, lay.M,
                              c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[9], len(lay.A_dep_flat), c[10], c[11],
                              len(lay.B_dep_flat), c[12], flags)


def test_neg_efe_bwd_validation():
    lay = _efe_layout_args()
    op = "efe_ffi bwd: "
    assert _efe_bwd_call(lay) == _lib.B2_OK, _lib.last_error()
    assert _efe_bwd_call(lay, Bn=-1) == _lib.B2_ERR_INVALID_ARGUMENT
    assert _lib.last_error() == op + "negative Bn"
    # the adjoint covers the utility and state-information-gain terms only
    for flag in (_lib.FLAG_USE_PARAM_INFO_GAIN, _lib.FLAG_USE_INDUCTIVE):
        assert _efe_bwd_call(lay, flags=3 | flag) == _lib.B2_ERR_UNSUPPORTED
        assert _lib.last_error() == op + "only the utility and state-information-gain terms"
    assert _efe_bwd_call(lay, Bn=2, counts={"dG": 5}) == _lib.B2_ERR_INVALID_ARGUMENT
    assert _lib.last_error() == op + "d_neg_efe element_count = 5, expected 6"
    assert _efe_bwd_call(lay, Bn=2) == _lib.B2_ERR_INVALID_ARGUMENT
    assert _lib.last_error() == op + "null buffer"


def test_neg_efe_cached_needs_its_cache_and_shares_the_validation():
    """b2_neg_efe_cached is b2_neg_efe plus a caller-owned operand cache: a
    missing cache is an error; the rest of the validation and the empty-batch
    no-op are b2_neg_efe's."""
    lib = _lib.load()
    lay = _efe_layout_args()
    c = lay._c
    P = 3
    cache = (ctypes.c_uint8 * 256)()
    valid = ctypes.c_int32(0)

    def call(Bn, A_count, cache_ptr, valid_ptr):
        return lib.b2_neg_efe_cached(None, 1, P * lay.T * lay.F, 0, 1, Bn * lay.qs_offsets[-1], 1, A_count, 1,
                                     Bn * lay.B_offsets[-1], 1, Bn * lay.C_offsets[-1], 1, Bn * lay.I_offsets[-1], 1,
                                     0, 1, 0, 1, 1, 1, Bn * P, Bn, P, lay.T, lay.F, lay.M, c[0], c[1], c[2], c[3],
                                     c[4], c[5], c[6], c[7], c[8], c[9], len(lay.A_dep_flat), c[10], c[11],
                                     len(lay.B_dep_flat), c[12], 3, cache_ptr, 256, valid_ptr)

    assert call(0, 0, None, ctypes.byref(valid)) == _lib.B2_ERR_INVALID_ARGUMENT
    assert "null pack cache" in _lib.last_error()
    assert call(0, 0, cache, None) == _lib.B2_ERR_INVALID_ARGUMENT
    assert call(0, 0, cache, ctypes.byref(valid)) == _lib.B2_OK, _lib.last_error()
    assert valid.value == 0  # nothing packed for an empty batch
    assert call(0, 5, cache, ctypes.byref(valid)) == _lib.B2_ERR_INVALID_ARGUMENT
    assert "A element_count = 5, expected 0" in _lib.last_error()
