"""Sequence inference (MMP / VMP): the FP64 oracle against the golden fixtures
made by the reference's own ``run_mmp`` / ``run_vmp`` (``pymdp/algos.py:312-571``).
This pins the checker for a sequence-inference kernel; no kernel runs here."""

import numpy as np
import pytest

from conftest import load_golden, unpack
from oracle import mmp


def _deps(d, key):
    out, i = [], 0
    for n in d[key + "_len"]:
        out.append(d[key + "_flat"][i:i + n].tolist())
        i += n
    return out


@pytest.mark.parametrize("name", ["seq_mmp", "seq_mmp_index", "seq_vmp", "seq_vmp_index", "seq_mmp_bench",
                                  "seq_vmp_bench", "seq_mmp_rank3", "seq_vmp_t1"])
def test_oracle_matches_reference_fixture(name):
    d = load_golden(name)
    qs = mmp.run_sequence(str(d["kind"]), unpack(d, "A"), unpack(d, "B"), unpack(d, "obs"), unpack(d, "prior"),
                          _deps(d, "A_deps"), _deps(d, "B_deps"), num_iter=int(d["num_iter"]), tau=float(d["tau"]),
                          distr_obs=bool(d["distr"]))
    for got, want in zip(qs, unpack(d, "qs")):
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(got.sum(-1), 1.0, atol=1e-12)
