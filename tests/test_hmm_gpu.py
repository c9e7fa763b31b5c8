"""Exact single-factor HMM inference on the GPU through the C-ABI
(``b2_hmm_smoother``, ``b2_hmm_smoother_from_filtered``) against the golden
fixtures made by the reference's ``pymdp/algos.py`` / ``pymdp/inference.py``
and the FP64 oracle (``oracle/hmm.py``).

The kernels run the recurrences in FP64 on float32 inputs and round the
outputs to float32; the backward pass reads the float32 filtered marginals, as
the reference's smoother does. Tolerances: rtol 1e-5, atol 1e-6 on
probabilities; rtol 1e-6 on the log marginal likelihood."""

import numpy as np
import pytest
import torch

from conftest import load_golden, unpack
from oracle import hmm as oh

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-5, 1e-6
SCAN = ["hmm_scan_actions", "hmm_scan_distr", "hmm_scan_time_varying", "hmm_scan_T1", "hmm_scan_wide"]


def cuda(x, dtype=torch.float32):
    return torch.as_tensor(np.asarray(x), device="cuda").to(dtype).contiguous()


@pytest.mark.parametrize("name", SCAN)
def test_scan_matches_reference_fixture(name):
    from pymdp_b200 import hmm
    d = load_golden(name)
    A, obs = unpack(d, "A"), unpack(d, "obs")
    T, distr = int(d["T"]), bool(d["distr"])
    acts = cuda(d["actions"], torch.int32) if "actions" in d and T > 1 else None
    odt = torch.float32 if distr else torch.int32
    r = hmm.hmm_smoother([cuda(a) for a in A], [cuda(o, odt) for o in obs], cuda(d["prior"]), cuda(d["B"]),
                         actions=acts, distr_obs=distr,
                         want=("mll", "filtered", "predicted", "smoothed", "cond", "joint"))
    torch.cuda.synchronize()
    np.testing.assert_allclose(r["mll"].cpu().numpy(), d["mll"], rtol=1e-6)
    for k in ("filtered", "predicted", "smoothed", "cond"):
        np.testing.assert_allclose(r[k].cpu().numpy(), d[k], rtol=RTOL, atol=ATOL, err_msg=k)
    if T > 1:  # joint[t, j, i] = cond[t, j, i] * smoothed[t+1, j]
        np.testing.assert_allclose(r["joint"].cpu().numpy(), d["cond"] * d["smoothed"][:, 1:, :, None],
                                   rtol=RTOL, atol=ATOL)
    # the reference-named wrapper returns the same arrays
    mll, qs, ps, qss = hmm.run_exact_single_factor_hmm_scan(
        [cuda(o, odt) for o in obs], [cuda(a) for a in A], [cuda(d["B"])], [cuda(d["prior"])], actions=acts,
        distr_obs=distr)
    assert torch.equal(qs[0], r["smoothed"]) and torch.equal(ps[0], r["predicted"]) and torch.equal(qss[0], r["cond"])


def test_smoothing_exact_matches_reference_fixture():
    """Negative actions are identity transitions (invalid_action_mode="identity")."""
    from pymdp_b200 import hmm
    d = load_golden("hmm_smoothing_exact")
    sm, joint = hmm.smoothing_exact([cuda(d["filtered"])], [cuda(d["B"])], cuda(d["actions"], torch.int32))
    torch.cuda.synchronize()
    np.testing.assert_allclose(sm[0].cpu().numpy(), d["smoothed"], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(joint[0].cpu().numpy(), d["joint"], rtol=RTOL, atol=ATOL)


def test_smoother_from_filtered_matches_scan_fixture():
    from pymdp_b200 import hmm
    d = load_golden("hmm_scan_actions")
    sm, joint, cond, trans = hmm.hmm_smoother_from_filtered_colstoch(
        cuda(d["filtered"]), cuda(d["B"]), actions=cuda(d["actions"], torch.int32), return_trans_probs=True)
    torch.cuda.synchronize()
    np.testing.assert_allclose(sm.cpu().numpy(), d["smoothed"], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(cond.cpu().numpy(), d["cond"], rtol=RTOL, atol=ATOL)
    assert torch.equal(trans, joint.transpose(-1, -2))


def test_benchmark_size_identities_and_samples():
    """4096 agents, T = 64, K = 32, U = 4, two modalities: the joint's
    marginals are the smoothed marginals (summing out the next state, axis 2,
    gives step t; summing out the current state, axis 3, gives step t+1), the
    last smoothed marginal is the last filtered one, and sampled agents match
    the FP64 oracle."""
    from pymdp_b200 import hmm
    Bn, T, K, U, O = 4096, 64, 32, 4, [16, 8]
    g = torch.Generator(device="cuda").manual_seed(9)
    A = [torch.softmax(torch.randn((Bn, o, K), device="cuda", generator=g) * 2, dim=1) for o in O]
    B = torch.softmax(torch.randn((Bn, K, K, U), device="cuda", generator=g) * 2, dim=1)
    prior = torch.softmax(torch.randn((Bn, K), device="cuda", generator=g), dim=1)
    obs = [torch.randint(0, o, (Bn, T), device="cuda", generator=g, dtype=torch.int32) for o in O]
    acts = torch.randint(0, U, (Bn, T - 1), device="cuda", generator=g, dtype=torch.int32)
    r = hmm.hmm_smoother(A, obs, prior, B, actions=acts, distr_obs=False,
                         want=("mll", "filtered", "predicted", "smoothed", "joint"))
    torch.cuda.synchronize()
    sm, joint, filt = r["smoothed"].double(), r["joint"].double(), r["filtered"].double()
    assert torch.allclose(joint.sum(2), sm[:, :-1], atol=2e-5)
    assert torch.allclose(joint.sum(3), sm[:, 1:], atol=2e-5)
    assert torch.allclose(sm[:, -1], filt[:, -1], atol=1e-6)
    assert torch.allclose(sm.sum(-1), torch.ones_like(sm.sum(-1)), atol=1e-5)
    for b in (0, 1234, Bn - 1):
        mll, s, p, c, f = oh.run_exact_single_factor_hmm_scan(
            [o[b].cpu().numpy() for o in obs], [a[b].cpu().numpy() for a in A], [B[b].cpu().numpy()],
            [prior[b].cpu().numpy()], actions=acts[b].cpu().numpy(), distr_obs=False)
        np.testing.assert_allclose(r["mll"][b].item(), mll, rtol=1e-6)
        np.testing.assert_allclose(r["filtered"][b].cpu().numpy(), f, rtol=RTOL, atol=ATOL)
        np.testing.assert_allclose(r["smoothed"][b].cpu().numpy(), s[0], rtol=1e-4, atol=1e-5)
