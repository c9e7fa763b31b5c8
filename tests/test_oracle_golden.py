"""Pin the FP64 oracle against golden vectors produced by the reference's own
code (``pymdp/algos.py::run_factorized_fpi``, ``pymdp/control.py::
update_posterior_policies``; see ``tests/golden/make_golden.py``)."""

import numpy as np
import pytest

from conftest import deps_from, load_golden, unpack
from oracle import efe as oefe
from oracle import fpi as ofpi

FPI = ["fpi_plain", "fpi_single_factor", "fpi_rank123", "fpi_rank4", "fpi_orphan_factor",
       "fpi_cfg2", "fpi_large"]
EFE = ["efe_plain", "efe_mixed", "efe_bdeps", "efe_cfg3_t1", "efe_cfg3_small"]


@pytest.mark.parametrize("name", FPI)
def test_fpi_oracle_matches_reference(name):
    d = load_golden(name)
    deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    A = unpack(d, "A")
    prior = [p.astype(np.float64) for p in unpack(d, "prior")]
    qs_ref = unpack(d, "qs")
    qs = ofpi.run_fpi_batch([a.astype(np.float64) for a in A], d["obs"], prior, deps, int(d["num_iter"]))
    for f in range(len(qs)):
        np.testing.assert_allclose(qs[f], qs_ref[f], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("name", FPI)
def test_fpi_oracle_from_ll_matches_reference(name):
    d = load_golden(name)
    deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    ll = unpack(d, "ll")
    prior = unpack(d, "prior")
    qs_ref = unpack(d, "qs")
    for b in range(d["obs"].shape[0]):
        if len(prior) == 1:
            continue  # reference takes the one-pass branch before the FFI call
        qs = ofpi.fpi_from_ll([l[b] for l in ll], [ofpi.log_stable(p[b]) for p in prior], deps,
                              int(d["num_iter"]))
        for f in range(len(qs)):
            np.testing.assert_allclose(qs[f], qs_ref[f][b], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("name", EFE)
def test_efe_oracle_matches_reference(name):
    d = load_golden(name)
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    S, U, T = d["S"].tolist(), d["U"].tolist(), int(d["T"])
    pol = oefe.construct_policies(S, U, T)
    np.testing.assert_array_equal(pol, d["policies"])
    q_pi, G = oefe.update_posterior_policies(pol, unpack(d, "qs"), unpack(d, "A"), unpack(d, "B"),
                                             unpack(d, "C"), d["E"], A_deps, B_deps,
                                             gamma=float(d["gamma"]))
    np.testing.assert_allclose(G, d["G"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(q_pi, d["q_pi"], rtol=1e-10, atol=1e-300)
    np.testing.assert_array_equal(oefe.sample_policy(pol, q_pi), d["action"])


EFE_EXTRA = ["efe_pig", "efe_pigA", "efe_ind", "efe_all"]


def extra_terms(d):
    """Keyword arguments of the flag-gated terms stored in an extra golden case."""
    return dict(pA=unpack(d, "pA") if int(d["has_pA"]) else None,
                pB=unpack(d, "pB") if int(d["has_pB"]) else None,
                use_param_info_gain=bool(int(d["use_param_info_gain"])),
                I=unpack(d, "I"), use_inductive=bool(int(d["use_inductive"])),
                inductive_epsilon=float(d["eps"]))


@pytest.mark.parametrize("name", EFE_EXTRA)
def test_efe_oracle_extra_terms_match_reference(name):
    """Parameter information gain (pA / pB) and the inductive value, against
    the reference's own update_posterior_policies_inductive (control.py:795-963)."""
    d = load_golden(name)
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    S, U, T = d["S"].tolist(), d["U"].tolist(), int(d["T"])
    pol = oefe.construct_policies(S, U, T)
    np.testing.assert_array_equal(pol, d["policies"])
    q_pi, G = oefe.update_posterior_policies(pol, unpack(d, "qs"), unpack(d, "A"), unpack(d, "B"),
                                             unpack(d, "C"), d["E"], A_deps, B_deps,
                                             gamma=float(d["gamma"]), **extra_terms(d))
    np.testing.assert_allclose(G, d["G"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(q_pi, d["q_pi"], rtol=1e-10, atol=1e-300)
    np.testing.assert_array_equal(oefe.sample_policy(pol, q_pi), d["action"])


@pytest.mark.parametrize("name", ["fpi_bad_obs", "fpi_bad_obs_single"])
def test_fpi_oracle_out_of_range_observation_matches_reference(name):
    """An observation outside [0, O_m) is an all-zero one-hot in the reference
    (jax.nn.one_hot): that modality adds nothing (tests/golden/make_golden_edges.py)."""
    d = load_golden(name)
    deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    obs = d["obs"]
    assert ((obs < 0) | (obs >= d["O"][None, :])).any()
    qs = ofpi.run_fpi_batch([a.astype(np.float64) for a in unpack(d, "A")], obs,
                            [p.astype(np.float64) for p in unpack(d, "prior")], deps, int(d["num_iter"]))
    for f, q in enumerate(unpack(d, "qs")):
        np.testing.assert_allclose(qs[f], q, rtol=1e-12, atol=1e-14)


def test_efe_oracle_out_of_range_action_matches_reference():
    """Actions outside [0, U_f) are read as JAX's gather reads them (negative
    from the end, then clamped), as in the reference's B_f[..., u_f]."""
    d = load_golden("efe_bad_action")
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    pol = d["policies"]
    np.testing.assert_array_equal(oefe.jnp_index(pol, d["U"][None, None, :]), d["policies_as_read"])
    q_pi, G = oefe.update_posterior_policies(pol, unpack(d, "qs"), unpack(d, "A"), unpack(d, "B"), unpack(d, "C"),
                                             d["E"], A_deps, B_deps, gamma=float(d["gamma"]))
    np.testing.assert_allclose(G, d["G"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(q_pi, d["q_pi"], rtol=1e-10, atol=1e-300)


def test_multiaction_oracle_marginal_and_full_agree_on_product_policies():
    """For the full product policy set the "marginal" mode's outer product of
    action marginals and the "full" mode's sums coincide when q_pi factorises
    over the first-step actions; both sum to one."""
    S, U, T = [3, 2, 2], [3, 2, 1], 2
    pol = oefe.construct_policies(S, U, T)
    rng = np.random.default_rng(0)
    m = [rng.dirichlet(np.ones(u)) for u in U]
    q = np.array([np.prod([m[f][p[0, f]] for f in range(len(U))]) for p in pol]) / (len(pol) // int(np.prod(U)))
    full = oefe.multiaction_probabilities(q, pol, U, "full")
    marg = oefe.multiaction_probabilities(q, pol, U, "marginal")
    np.testing.assert_allclose(full, marg, rtol=1e-12)
    np.testing.assert_allclose(full.sum(), 1.0, rtol=1e-12)
