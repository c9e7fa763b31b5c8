"""FP64 CPU oracle for the FPI and EFE hot paths — TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy float64, the semantics of the reference's pure
JAX implementation (the branch its CI runs):

* ``oracle.fpi``  — ``pymdp/algos.py:88-155`` (``run_factorized_fpi``) and
  ``pymdp/maths.py:15-79,214-287`` (``log_stable``, log-likelihoods).
* ``oracle.efe``  — ``pymdp/control.py:198-509,604-690`` (expected states,
  expected observations, state info gain, utility, ``update_posterior_policies``)
  and ``pymdp/control.py:115-195`` (``construct_policies``, ``sample_policy``).
* ``oracle.fitting`` — the model-fitting action log-likelihood over trials
  (infer_states -> infer_policies -> multiaction_probabilities per trial).
* ``oracle.rollout`` — the closed-loop rollout of one agent (environment
  sampling, empirical prior, planning, action).
* ``oracle.learning`` — ``pymdp/learning.py:11-233`` and the filtering branch
  of ``Agent.infer_parameters`` (``pymdp/agent.py:416-620``).
* ``oracle.mmp`` — sequence inference, ``run_mmp`` / ``run_vmp``
  (``pymdp/algos.py:157-571``): the checker for a sequence-inference kernel.
* ``oracle.hmm`` — ``run_exact_single_factor_hmm_scan`` /
  ``hmm_smoother_from_filtered_colstoch`` (``pymdp/algos.py:959-1208``) and
  ``smoothing_exact`` (``pymdp/inference.py:595-634``).

Parity pin: the functions are checked against golden vectors produced by
running the reference's own Python code (``tests/golden/make_golden*.py``
through ``tests/golden/refshim.py``): ``tests/test_oracle_golden.py``,
``tests/test_learning_cpu.py``, ``tests/test_hmm_cpu.py``,
``tests/test_seq_oracle_cpu.py``. The same
functions, run on a spawned process pool over the host cores, are the timed
CPU baseline of ``bench.py``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker / the timed CPU
reference. The product path (``pymdp_b200``) never imports it.
"""

from . import fpi, efe  # noqa: F401
