"""Exact single-factor HMM inference on the CPU: the FP64 oracle against the
golden fixtures made by the reference's own ``pymdp/algos.py`` /
``pymdp/inference.py``, and the C-ABI's argument checks (no kernel runs)."""

import ctypes

import numpy as np
import pytest

from conftest import load_golden, unpack
from oracle import hmm as oh
from pymdp_b200 import _lib

SCAN = ["hmm_scan_actions", "hmm_scan_distr", "hmm_scan_time_varying", "hmm_scan_T1", "hmm_scan_wide"]


@pytest.mark.parametrize("name", SCAN)
def test_oracle_scan_matches_reference_fixture(name):
    d = load_golden(name)
    A, obs = unpack(d, "A"), unpack(d, "obs")
    T = int(d["T"])
    for b in range(int(d["Bn"])):
        acts = d["actions"][b] if "actions" in d and T > 1 else None
        mll, sm, pred, cond, filt = oh.run_exact_single_factor_hmm_scan(
            [o[b] for o in obs], [a[b] for a in A], [d["B"][b]], [d["prior"][b]], actions=acts,
            distr_obs=bool(d["distr"]))
        np.testing.assert_allclose(mll, d["mll"][b], rtol=1e-12)
        np.testing.assert_allclose(filt, d["filtered"][b], rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(pred[0], d["predicted"][b], rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(sm[0], d["smoothed"][b], rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(cond[0], d["cond"][b], rtol=1e-10, atol=1e-14)


def test_oracle_smoothing_exact_matches_reference_fixture():
    d = load_golden("hmm_smoothing_exact")
    for b in range(int(d["Bn"])):
        sm, joint = oh.smoothing_exact([d["filtered"][b]], [d["B"][b]], d["actions"][b])
        np.testing.assert_allclose(sm[0], d["smoothed"][b], rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(joint[0], d["joint"][b], rtol=1e-10, atol=1e-14)


def test_oracle_joint_marginals_are_consistent():
    """Size-independent identities the GPU tests use at full size: the joint's
    marginals are the smoothed marginals (summing out the next state gives step
    t, summing out the current state gives step t+1), and the last smoothed
    marginal is the last filtered one."""
    d = load_golden("hmm_scan_wide")
    A, obs = unpack(d, "A"), unpack(d, "obs")
    mll, sm, pred, cond, filt = oh.run_exact_single_factor_hmm_scan(
        [o[0] for o in obs], [a[0] for a in A], [d["B"][0]], [d["prior"][0]], actions=d["actions"][0],
        distr_obs=False)
    B_seq = oh.select_transitions(d["B"][0], d["actions"][0], int(d["T"]))
    s, joint, _ = oh.smoother_from_filtered(filt, B_seq)
    np.testing.assert_allclose(joint.sum(1), s[:-1], atol=1e-12)
    np.testing.assert_allclose(joint.sum(2), s[1:], atol=1e-12)
    np.testing.assert_allclose(s[-1], filt[-1], atol=1e-15)


def test_hmm_abi_validation():
    lib = _lib.load()
    O = (ctypes.c_int64 * 1)(4)
    fake = 0x1000
    # K above the build's limit
    rc = lib.b2_hmm_smoother(None, fake, 4 * 200, 0, O, 1, fake, 0, 3, fake, 200, fake, 200 * 200 * 2, 0, 2, fake, 2,
                             0, 1, 3, 200, fake, fake, 0, 0, 0, 0)
    assert rc == _lib.B2_ERR_UNSUPPORTED
    # B count mismatch (stationary with U = 2, shared)
    rc = lib.b2_hmm_smoother(None, fake, 4 * 5, 0, O, 1, fake, 0, 3, fake, 5, fake, 5 * 5 * 2 - 1, 0, 2, fake, 2,
                             0, 1, 3, 5, fake, fake, 0, 0, 0, 0)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and b"B_count" in lib.b2_last_error()
    # actions required when B has several actions
    rc = lib.b2_hmm_smoother(None, fake, 4 * 5, 0, O, 1, fake, 0, 3, fake, 5, fake, 5 * 5 * 2, 0, 2, None, 0,
                             0, 1, 3, 5, fake, fake, 0, 0, 0, 0)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and b"actions" in lib.b2_last_error()
    # bad action mode
    rc = lib.b2_hmm_smoother_from_filtered(None, fake, 15, fake, 50, 0, 2, fake, 2, 5, 1, 3, 5, fake, 0, 0)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT
    # an empty batch is a valid no-op
    rc = lib.b2_hmm_smoother_from_filtered(None, fake, 0, fake, 50, 0, 2, fake, 0, 1, 0, 3, 5, fake, 0, 0)
    assert rc == _lib.B2_OK


def test_transition_layout_rules():
    """The host classifies B as the reference's per-sequence shapes plus an
    optional batch axis (no device work)."""
    import torch

    from pymdp_b200.hmm import _transitions
    Bn, T, K = 3, 5, 4
    # action axis: shared (K, K, U) or batched (Bn, K, K, U), actions reshaped to (Bn, T-1)
    t, batched, U, a = _transitions(torch.zeros(K, K, 2), np.zeros((Bn, T - 1, 1), np.int64), Bn, T, K)
    assert (batched, U, tuple(a.shape), a.dtype) == (0, 2, (Bn, T - 1), torch.int32)
    t, batched, U, a = _transitions(torch.zeros(Bn, K, K, 2), np.zeros((Bn, T - 1)), Bn, T, K)
    assert (batched, U) == (1, 2)
    # stationary without actions: one action
    t, batched, U, a = _transitions(torch.zeros(K, K), None, Bn, T, K)
    assert (batched, U, a, tuple(t.shape)) == (0, 1, None, (K, K, 1))
    t, batched, U, a = _transitions(torch.zeros(Bn, K, K), None, Bn, T, K)
    assert (batched, U, tuple(t.shape)) == (1, 1, (Bn, K, K, 1))
    # time-varying (T-1, K, K), shared or batched
    t, batched, U, a = _transitions(torch.zeros(T - 1, K, K), None, Bn, T, K)
    assert (batched, U) == (0, 0)
    t, batched, U, a = _transitions(torch.zeros(Bn, T - 1, K, K), None, Bn, T, K)
    assert (batched, U) == (1, 0)
    # several actions and no action history: the reference's error
    with pytest.raises(ValueError):
        _transitions(torch.zeros(K, K, 3), None, Bn, T, K)
    # one observation: no transition is taken, any action axis is accepted
    t, batched, U, a = _transitions(torch.zeros(K, K, 3), None, Bn, 1, K)
    assert U == 3
