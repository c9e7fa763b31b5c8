"""pymdp_b200 — B200-native (sm_100a) FPI and EFE hot paths of pymdp.

* ``pymdp_b200.ffi``   — drop-in mirror of ``pymdp.ffi`` (``fpi_ffi``,
  ``neg_efe_all_policies_ffi``, gates, flatten helpers) over the C-ABI.
* ``pymdp_b200.Agent`` — ``infer_states`` / ``infer_policies`` /
  ``sample_action`` with the reference's signatures.
* ``include/pymdp_b200.h`` — the C-ABI itself (``libpymdp_b200.so``).
"""

from .control import construct_policies  # noqa: F401


def __getattr__(name):
    # torch-backed modules load lazily so the C-ABI can be used without torch
    import importlib

    if name == "Agent":
        return importlib.import_module(".agent", __name__).Agent
    if name in ("ffi", "agent"):
        return importlib.import_module("." + name, __name__)
    raise AttributeError(name)
