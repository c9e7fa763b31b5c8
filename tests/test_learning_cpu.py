"""Online Dirichlet learning on the CPU: the FP64 oracle against the golden
fixtures made by the reference's own ``pymdp/learning.py``, the batch-level
gating of ``Agent.infer_parameters`` (``pymdp/agent.py:480-500``), and the
C-ABI's argument checks (no kernel runs)."""

import ctypes

import numpy as np
import pytest

from conftest import load_golden, unpack
from oracle import learning as ol
from pymdp_b200 import _lib, ffi


def _deps(d):
    out, i = [], 0
    for n in d["deps_len"]:
        out.append(d["deps_flat"][i:i + n].tolist())
        i += n
    return out


@pytest.mark.parametrize("name", ["learn_A_full", "learn_A_window", "learn_A_cat", "learn_A_long"])
def test_oracle_obs_model_matches_reference_fixture(name):
    d = load_golden(name)
    A, pA, obs, qs = unpack(d, "A"), unpack(d, "pA"), unpack(d, "obs"), unpack(d, "qs")
    none = d["none_mask"]
    deps = _deps(d)
    for b in range(int(d["Bn"])):
        qA, EA = ol.update_obs_likelihood_dirichlet(
            [None if none[m] else p[b] for m, p in enumerate(pA)], [a[b] for a in A], [o[b] for o in obs],
            [q[b] for q in qs], deps, d["O"].tolist(), lr=d["lr"][b], categorical_obs=bool(d["categorical"]))
        for m in range(len(A)):
            ref_q = d[f"qA{m}"][b]
            np.testing.assert_allclose(pA[m][b] if qA[m] is None else qA[m], ref_q, rtol=1e-13, atol=0)
            np.testing.assert_allclose(EA[m], d[f"EA{m}"][b], rtol=1e-13, atol=1e-300)


@pytest.mark.parametrize("name", ["learn_B_online", "learn_B_window", "learn_B_long"])
def test_oracle_transition_model_matches_reference_fixture(name):
    d = load_golden(name)
    B, pB, qs = unpack(d, "B"), unpack(d, "pB"), unpack(d, "qs")
    deps = _deps(d)
    act = d["actions"]
    S, U = d["S"].tolist(), d["U"].tolist()
    mask = int(d["factor_mask"])
    out = ol.infer_parameters(None, None, pB, B, qs, None, act, None, deps, None, U, learn_A=False, learn_B=True,
                              lr_pB=d["lr"])
    for f in range(len(S)):
        if not (mask >> f) & 1:
            continue  # the fixture's factors_to_update: checked below through the single-agent call
        np.testing.assert_allclose(out[2][f], d[f"qB{f}"], rtol=1e-13, atol=0)
        np.testing.assert_allclose(out[3][f], d[f"EB{f}"], rtol=1e-13, atol=1e-300)
    fts = "all" if mask == (1 << len(S)) - 1 else [f for f in range(len(S)) if (mask >> f) & 1]
    valid = np.all(act >= 0, axis=-1).astype(np.float64)
    for b in range(int(d["Bn"])):
        m = valid[b][:, None]
        joints = [[qs[f][b, 1:] * m] + [qs[x][b, :-1] * m for x in deps[f]] for f in range(len(S))]
        qB, EB = ol.update_state_transition_dirichlet([p[b] for p in pB], [x[b] for x in B], joints, act[b], U,
                                                      lr=d["lr"][b], factors_to_update=fts)
        for f in range(len(S)):
            np.testing.assert_allclose(qB[f], d[f"qB{f}"][b], rtol=1e-13, atol=0)
            np.testing.assert_allclose(EB[f], d[f"EB{f}"][b], rtol=1e-13, atol=1e-300)


def test_oracle_gating_skips_B_without_a_valid_transition():
    """agent.py:486-500: no agent with a valid transition (or T = 1) keeps pB
    and B as they are (B is not renormalised)."""
    d = load_golden("learn_B_online")
    B, pB, qs = unpack(d, "B"), unpack(d, "pB"), unpack(d, "qs")
    B = [x * 1.5 for x in B]  # deliberately not E[pB]
    deps = _deps(d)
    bad = np.full_like(d["actions"], -1)
    out = ol.infer_parameters(None, None, pB, B, qs, None, bad, None, deps, None, d["U"].tolist(), learn_A=False)
    assert all(o is x for o, x in zip(out[3], B))
    one = [q[:, :1] for q in qs]
    out = ol.infer_parameters(None, None, pB, B, one, None, d["actions"], None, deps, None, d["U"].tolist(),
                              learn_A=False)
    assert all(o is x for o, x in zip(out[3], B))
    # one valid transition anywhere in the batch renormalises every agent's B
    some = bad.copy()
    some[0, 0] = 0
    out = ol.infer_parameters(None, None, pB, B, qs, None, some, None, deps, None, d["U"].tolist(), learn_A=False)
    for f in range(len(B)):
        np.testing.assert_allclose(out[3][f][1], ol.dirichlet_expected_value(pB[f][1]), rtol=1e-15)


def test_oracle_mass_conservation():
    """Each index observation adds lr * sum_k prod_f q_f = lr to a modality's
    counts (beliefs normalised, here to float32 rounding) — the
    size-independent property the GPU tests use at full size."""
    d = load_golden("learn_A_window")
    A, pA, obs, qs = unpack(d, "A"), unpack(d, "pA"), unpack(d, "obs"), unpack(d, "qs")
    deps = _deps(d)
    T = int(d["T"])
    for b in range(int(d["Bn"])):
        qA, _ = ol.update_obs_likelihood_dirichlet([p[b] for p in pA], [a[b] for a in A], [o[b] for o in obs],
                                                   [q[b] for q in qs], deps, d["O"].tolist(), lr=d["lr"][b])
        for m in range(len(A)):
            n_in = int(np.sum((obs[m][b] >= 0) & (obs[m][b] < d["O"][m])))
            assert abs((qA[m] - pA[m][b]).sum() - d["lr"][b] * n_in) < 1e-6 * T


def test_learning_abi_validation():
    """Both entry points reject inconsistent layouts before any device work."""
    lib = _lib.load()
    S = (ctypes.c_int64 * 2)(4, 3)
    O = (ctypes.c_int64 * 1)(5)
    qo = (ctypes.c_int64 * 3)(0, 4, 7)
    Ao = (ctypes.c_int64 * 2)(0, 5 * 12)
    dep = (ctypes.c_int64 * 2)(0, 1)
    do = (ctypes.c_int64 * 2)(0, 2)
    fake = 0x1000
    # A_offsets inconsistent with O * K
    bad = (ctypes.c_int64 * 2)(0, 59)
    rc = lib.b2_update_obs_likelihood_dirichlet(None, fake, fake, 2 * 59, fake, 0, 2, fake, 2 * 7, fake, 1, 2, 1,
                                                2, 1, S, O, qo, bad, dep, 2, do, 1)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and b"A_offsets" in lib.b2_last_error()
    # obs count
    rc = lib.b2_update_obs_likelihood_dirichlet(None, fake, fake, 2 * 60, fake, 0, 3, fake, 2 * 7, fake, 1, 2, 1,
                                                2, 1, S, O, qo, Ao, dep, 2, do, 1)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and b"obs_count" in lib.b2_last_error()
    # dependency out of range
    dep_bad = (ctypes.c_int64 * 2)(0, 2)
    rc = lib.b2_update_obs_likelihood_dirichlet(None, fake, fake, 2 * 60, fake, 0, 2, fake, 2 * 7, fake, 1, 2, 1,
                                                2, 1, S, O, qo, Ao, dep_bad, 2, do, 1)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and b"dependency" in lib.b2_last_error()
    # an empty modality mask is a valid no-op
    rc = lib.b2_update_obs_likelihood_dirichlet(None, fake, fake, 2 * 60, fake, 0, 2, fake, 2 * 7, fake, 1, 2, 1,
                                                2, 1, S, O, qo, Ao, dep, 2, do, 0)
    assert rc == _lib.B2_OK
    # transition model: B_offsets must be S_f * K_f * U_f
    U = (ctypes.c_int64 * 2)(2, 1)
    Bo = (ctypes.c_int64 * 3)(0, 4 * 4 * 2 - 1, 4 * 4 * 2 - 1 + 3 * 3 * 1)
    bdep = (ctypes.c_int64 * 2)(0, 1)
    bdo = (ctypes.c_int64 * 3)(0, 1, 2)
    rc = lib.b2_update_state_transition_dirichlet(None, fake, fake, 2 * 40, fake, 2 * 2 * 7, fake, 2 * 1 * 2, fake, 1,
                                                  fake, 2, 2, 2, S, U, qo, Bo, bdep, 2, bdo, 3)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and b"B_offsets" in lib.b2_last_error()
    Bo = (ctypes.c_int64 * 3)(0, 32, 41)
    rc = lib.b2_update_state_transition_dirichlet(None, fake, fake, 2 * 41, fake, 2 * 2 * 7, fake, 3, fake, 1,
                                                  fake, 2, 2, 2, S, U, qo, Bo, bdep, 2, bdo, 3)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and b"actions_count" in lib.b2_last_error()
    # a window of one time step has no transition: valid no-op
    rc = lib.b2_update_state_transition_dirichlet(None, fake, fake, 2 * 41, fake, 2 * 1 * 7, fake, 0, fake, 1,
                                                  fake, 2, 1, 2, S, U, qo, Bo, bdep, 2, bdo, 3)
    assert rc == _lib.B2_OK


def test_layout_learning_wrappers_exist():
    lay = ffi.EfeLayout([4, 3], [5], [2, 1], 1, [[0, 1]], [[0], [1]])
    assert callable(lay.learn_A) and callable(lay.learn_B)


def test_oracle_transition_model_from_joints_matches_reference_fixture():
    """The smoothing algorithms' form: pB learns from given pairwise joints
    (learning.py:153, a joint array per factor) — the checker for a
    joint-input transition update."""
    d = load_golden("learn_B_joint")
    for b in range(int(d["Bn"])):
        qb, eb = ol.update_state_transition_from_joint(d["pB"][b], d["joint"][b], d["actions"][b][:, 0],
                                                       int(d["U"]), lr=d["lr"][b])
        np.testing.assert_allclose(qb, d["qB"][b], rtol=1e-13, atol=0)
        np.testing.assert_allclose(eb, d["EB"][b], rtol=1e-13, atol=1e-300)
