"""Policy construction (host-side, integer bookkeeping only).

``construct_policies`` follows ``pymdp/control.py:152-195``: the policy
matrix enumerates ``itertools.product`` over ``num_controls * policy_len``
and reshapes each tuple to ``(policy_len, num_factors)``.
"""

from __future__ import annotations

import itertools
from typing import Sequence

import numpy as np


def construct_policies(num_states: Sequence[int], num_controls: Sequence[int] | None = None, policy_len: int = 1,
                       control_fac_idx: Sequence[int] | None = None) -> np.ndarray:
    """``(P, policy_len, F)`` int32 policy matrix in the reference's order."""
    F = len(num_states)
    if control_fac_idx is None:
        if num_controls is not None:
            control_fac_idx = [f for f, n in enumerate(num_controls) if n > 1]
        else:
            control_fac_idx = list(range(F))
    if num_controls is None:
        num_controls = [num_states[c] if c in control_fac_idx else 1 for c in range(F)]
    x = list(num_controls) * policy_len
    pols = list(itertools.product(*[range(int(i)) for i in x]))
    return np.asarray(pols, dtype=np.int32).reshape(len(pols), policy_len, F)


def generate_I_matrix(H: Sequence, B: Sequence, threshold: float, depth: int) -> list:
    """Backward reachability matrices of the inductive term
    (``pymdp/control.py:965-1019``), host-side set-up for one agent.

    ``H[f]``: ``(S_f,)`` goal indicator; ``B[f]``: ``(S_f, S_f, U_f)``
    (factor-local dynamics). Row ``i`` of ``I[f]`` marks the states that can
    still reach the goal set after ``i`` backward steps, through transitions
    whose probability exceeds ``threshold`` under some action.
    """
    if depth < 1:
        raise ValueError("`depth` must be >= 1")
    out = []
    for h, b in zip(H, B):
        b = np.asarray(b, np.float64)
        h = np.asarray(h, np.float64)
        if b.ndim != 3 or b.shape[0] != b.shape[1]:
            raise ValueError("generate_I_matrix needs factor-local B of shape (S, S, U)")
        reach = ((b > threshold).sum(axis=-1) > 0).astype(np.float64)  # [next, prev]
        pred = reach.T
        rows = [h]
        for _ in range(depth - 1):
            rows.append((pred @ rows[-1] > 0).astype(np.float64))
        out.append(np.stack(rows, axis=0).astype(np.float32))
    return out
