"""The reference's own CPU FFI kernels (NegEfeCpu, FpiCpu; compiled from the
reference's sources by oracle/ref_build.py into oracle/_ref) against the
golden fixtures made by the reference's JAX-semantics Python code. This pins
the CPU timing baseline to the same computation as the oracle and the GPU
path. The reference CPU kernels are FP32 (-ffast-math) and FPI stops early at
max |d log q| < 1e-5, hence the FP32-level tolerances here."""

import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, deps_from, load_golden, unpack


@pytest.fixture(scope="module")
def refcpu():
    from oracle import ref_build
    if not ref_build.build():
        pytest.skip("reference sources absent and no prebuilt oracle/_ref library")
    from oracle import refcpu as rc
    return rc


def _flat(xs, n):
    return np.concatenate([np.asarray(x, np.float32).reshape(n, -1) for x in xs], axis=1)


@pytest.mark.parametrize("name", ["efe_plain", "efe_mixed", "efe_bdeps", "efe_cfg3_t1", "efe_cfg3_small"])
def test_reference_neg_efe_cpu_matches_fixtures(refcpu, name):
    d = load_golden(name)
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    qs, A, B, C = unpack(d, "qs"), unpack(d, "A"), unpack(d, "B"), unpack(d, "C")
    pol = d["policies"]
    T = pol.shape[1]
    S, O, U = [q.shape[-1] for q in qs], [a.shape[0] for a in A], [b.shape[-1] for b in B]
    C = [np.broadcast_to(c, (T, c.shape[-1])) if c.ndim == 1 else c for c in C]
    spans = refcpu.efe_spans(S, O, U, T, A_deps, B_deps)
    G = refcpu.neg_efe_cpu(pol, _flat(qs, 1), _flat(A, 1), _flat(B, 1), _flat(C, 1),
                           np.zeros((1, sum(S)), np.float32), spans)
    np.testing.assert_allclose(G[0], d["G"], rtol=2e-6, atol=1e-6)


def test_reference_neg_efe_cpu_batched_form(refcpu):
    """The broadcast_all form ([Bn, P, T, F] policies) gives each agent its
    own G, equal to single-agent calls."""
    d = load_golden("efe_mixed")
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    qs, A, B, C = unpack(d, "qs"), unpack(d, "A"), unpack(d, "B"), unpack(d, "C")
    pol = d["policies"]
    T = pol.shape[1]
    S, O, U = [q.shape[-1] for q in qs], [a.shape[0] for a in A], [b.shape[-1] for b in B]
    C = [np.broadcast_to(c, (T, c.shape[-1])) if c.ndim == 1 else c for c in C]
    spans = refcpu.efe_spans(S, O, U, T, A_deps, B_deps)
    rng = np.random.default_rng(0)
    qs2 = [np.stack([q, rng.dirichlet(np.ones(q.shape[-1]))]) for q in qs]
    args = [_flat(x, 2) for x in ([np.stack([a, a]) for a in A], [np.stack([b, b]) for b in B],
                                  [np.stack([c, c]) for c in C])]
    G = refcpu.neg_efe_cpu(np.stack([pol, pol]), _flat(qs2, 2), *args, np.zeros((2, sum(S)), np.float32), spans)
    np.testing.assert_allclose(G[0], d["G"], rtol=2e-6, atol=1e-6)
    G1 = refcpu.neg_efe_cpu(pol, _flat([q[1] for q in qs2], 1), _flat(A, 1), _flat(B, 1), _flat(C, 1),
                            np.zeros((1, sum(S)), np.float32), spans)
    np.testing.assert_allclose(G[1], G1[0], rtol=1e-6, atol=1e-7)


FPI_LL = [p for p in sorted(glob.glob(os.path.join(GOLDEN, "fpi_*.npz"))) if "ll0" in np.load(p).files]


@pytest.mark.parametrize("path", FPI_LL, ids=os.path.basename)
def test_reference_fpi_cpu_matches_fixtures(refcpu, path):
    d = load_golden(os.path.basename(path)[:-4])
    S = [int(s) for s in d["S"]]
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    ll, prior = unpack(d, "ll"), unpack(d, "prior")
    n = ll[0].shape[0]
    K = [int(np.prod(x.shape[1:])) for x in ll]
    lp = np.concatenate([np.log(np.maximum(p, np.finfo(np.float64).eps)) for p in prior], axis=1)
    q = refcpu.fpi_cpu(_flat(ll, n), lp, S, np.cumsum([0] + K), A_deps, int(d["num_iter"]))
    np.testing.assert_allclose(q, np.concatenate(unpack(d, "qs"), axis=1), rtol=0, atol=1e-5)


def test_reference_cpu_errors_are_reported(refcpu):
    d = load_golden("efe_plain")
    A_deps = deps_from(d["A_dep_flat"], d["A_dep_offsets"])
    B_deps = deps_from(d["B_dep_flat"], d["B_dep_offsets"])
    qs, A, B, C = unpack(d, "qs"), unpack(d, "A"), unpack(d, "B"), unpack(d, "C")
    S, O, U = [q.shape[-1] for q in qs], [a.shape[0] for a in A], [b.shape[-1] for b in B]
    spans = refcpu.efe_spans(S, O, U, 1, A_deps, B_deps)
    with pytest.raises(ValueError, match="efe_ffi: A element_count = 47, expected 48"):
        refcpu.neg_efe_cpu(d["policies"], _flat(qs, 1), _flat(A, 1)[:, :-1], _flat(B, 1),
                           _flat([np.atleast_2d(c) for c in C], 1), np.zeros((1, sum(S)), np.float32), spans)
