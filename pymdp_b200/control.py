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
