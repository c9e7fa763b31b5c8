"""FP64 CPU oracle for the FPI and EFE hot paths — TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy float64, the semantics of the reference's pure
JAX implementation (the branch its CI runs):

* ``oracle.fpi``  — ``pymdp/algos.py:88-155`` (``run_factorized_fpi``) and
  ``pymdp/maths.py:15-79,214-287`` (``log_stable``, log-likelihoods).
* ``oracle.efe``  — ``pymdp/control.py:198-509,604-690`` (expected states,
  expected observations, state info gain, utility, ``update_posterior_policies``)
  and ``pymdp/control.py:115-195`` (``construct_policies``, ``sample_policy``).
* ``oracle.port`` — a plain C restatement of the same FP64 math with OpenMP
  over agents (``oracle/port.c``), used as the timed host-CPU baseline.

Parity pin: every function here is checked against golden vectors produced
by running the reference's own ``pymdp/algos.py`` / ``pymdp/control.py`` code
(``tests/golden/make_golden.py``), see ``tests/test_oracle_golden.py``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker / the timed CPU
reference. The product path (``pymdp_b200``) never imports it.
"""

from . import fpi, efe  # noqa: F401
