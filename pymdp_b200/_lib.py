"""ctypes binding of ``libpymdp_b200.so`` (the C-ABI in ``include/pymdp_b200.h``).

There is no fallback: if the library cannot be loaded every entry point
raises. Mirrors the role of the reference's library loader
(``pymdp/ffi/_core.py:41-80``), including the ``PYMDP_B200_LIB`` override
(the reference's is ``PYMDP_FFI_LIB``).
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_float, c_int32, c_int64, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PYMDP_B200_LIB", os.path.join(HERE, "libpymdp_b200.so"))

B2_OK = 0
B2_ERR_INVALID_ARGUMENT = 1
B2_ERR_UNSUPPORTED = 2
B2_ERR_CUDA = 3
B2_ERR_NO_DEVICE = 4

FLAG_USE_UTILITY = 1 << 0
FLAG_USE_STATES_INFO_GAIN = 1 << 1
FLAG_USE_INDUCTIVE = 1 << 2
FLAG_USE_PARAM_INFO_GAIN = 1 << 3
FLAG_MODEL_PARAMS_STATIC = 1 << 4
FLAG_POLICY_TREE = 1 << 5
FLAG_FACTORED = 1 << 6
PRECISION_SHIFT = 8
PRECISIONS = {"fp32": 0, "tf32x3": 1, "bf16": 2}

MAX_DEP_RANK = 8
MAX_FACTORS = 16
MAX_MODALITIES = 32
NOALLOC_SCRATCH_BYTES = 16 << 20


class B2Error(RuntimeError):
    """A failing C-ABI call; ``code`` is the B2_ERR_* status."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class UnsupportedError(B2Error, NotImplementedError):
    pass


class InvalidArgumentError(B2Error, ValueError):
    pass


_P64 = POINTER(c_int64)
_PF = c_void_p  # device float pointers are passed as raw addresses
_SIGS = {
    "b2_last_error": (ctypes.c_char_p, []),
    "b2_abi_version": (c_int32, []),
    "b2_capabilities": (c_int32, []),
    "b2_launch_count": (c_uint64, []),
    "b2_device_error": (c_int32, []),
    "b2_fpi": (c_int32, [c_void_p, _PF, c_int64, _PF, c_int64, _PF, c_int64, _P64, c_int64, _P64, c_int64,
                         _P64, c_int64, _P64, c_int64, _P64, c_int64, c_int32]),
    "b2_fpi_obs": (c_int32, [c_void_p, _PF, c_int64, _P64, c_int64, _P64, c_int64, c_void_p, _PF, _PF,
                             c_int64, _P64, c_int64, _P64, c_int64, _P64, c_int64, c_int32]),
    "b2_neg_efe": (c_int32, [c_void_p, c_void_p, c_int64, c_int32, _PF, c_int64, _PF, c_int64, _PF, c_int64,
                             _PF, c_int64, _PF, c_int64, _PF, c_int64, _PF, c_int64, _PF, c_int64, _PF,
                             c_int64, c_int64, c_int64, c_int64, c_int64, c_int64, _P64, _P64, _P64, _P64,
                             _P64, _P64, _P64, _P64, _P64, _P64, c_int64, _P64, _P64, c_int64, _P64,
                             c_int32]),
    "b2_neg_efe_noalloc": (c_int32, [c_void_p, c_void_p, c_int64, c_int32, _PF, c_int64, _PF, c_int64, _PF,
                                     c_int64, _PF, c_int64, _PF, c_int64, _PF, c_int64, _PF, c_int64, _PF,
                                     c_int64, _PF, c_int64, c_int64, c_int64, c_int64, c_int64, c_int64, _P64,
                                     _P64, _P64, _P64, _P64, _P64, _P64, _P64, _P64, _P64, c_int64, _P64, _P64,
                                     c_int64, _P64, c_int32]),
    "b2_neg_efe_bwd": (c_int32, [c_void_p, c_void_p, c_int64, c_int32, _PF, c_int64, _PF, c_int64, _PF, c_int64,
                                 _PF, c_int64, _PF, c_int64, _PF, _PF, _PF, _PF, c_int64, c_int64, c_int64, c_int64,
                                 c_int64, _P64, _P64, _P64, _P64, _P64, _P64, _P64, _P64, c_int64, _P64, _P64,
                                 c_int64, _P64, c_int32]),
    "b2_fpi_obs_bwd": (c_int32, [c_void_p, _PF, c_int64, _P64, c_int64, _P64, c_int64, c_void_p, _PF, _PF, _PF,
                                 _PF, c_int64, _P64, c_int64, _P64, c_int64, _P64, c_int64, c_int32]),
    "b2_policy_posterior": (c_int32, [c_void_p, _PF, _PF, c_int32, _PF, c_int32, _PF, c_int64, c_int64]),
    "b2_select_action": (c_int32, [c_void_p, _PF, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_int64]),
    "b2_neg_efe_cached": (c_int32, [c_void_p, c_void_p, c_int64, c_int32, _PF, c_int64, _PF, c_int64, _PF, c_int64,
                                    _PF, c_int64, _PF, c_int64, _PF, c_int64, _PF, c_int64, _PF, c_int64, _PF,
                                    c_int64, c_int64, c_int64, c_int64, c_int64, c_int64, _P64, _P64, _P64, _P64,
                                    _P64, _P64, _P64, _P64, _P64, _P64, c_int64, _P64, _P64, c_int64, _P64,
                                    c_int32, c_void_p, c_int64, POINTER(c_int32)]),
    "b2_neg_efe_pack_bytes": (c_int32, [c_int64, c_int64, c_int64, c_int64, c_int64, _P64, _P64, _P64, _P64, _P64,
                                        _P64, _P64, _P64, _P64, _P64, c_int64, _P64, _P64, c_int64, _P64, c_int32,
                                        POINTER(c_int64)]),
    "b2_sample_action": (c_int32, [c_void_p, _PF, c_void_p, _P64, c_void_p, c_int64, c_int64, c_int64, c_int64,
                                   c_int32, c_int32, _PF, c_int32, c_uint64]),
    "b2_update_obs_likelihood_dirichlet": (c_int32, [c_void_p, _PF, _PF, c_int64, c_void_p, _PF, c_int64, _PF,
                                                     c_int64, _PF, c_int32, c_int64, c_int64, c_int64, c_int64,
                                                     _P64, _P64, _P64, _P64, _P64, c_int64, _P64, c_int64]),
    "b2_update_state_transition_dirichlet": (c_int32, [c_void_p, _PF, _PF, c_int64, _PF, c_int64, c_void_p,
                                                       c_int64, _PF, c_int32, c_void_p, c_int64, c_int64, c_int64,
                                                       _P64, _P64, _P64, _P64, _P64, c_int64, _P64, c_int64]),
    "b2_update_state_transition_from_joint": (c_int32, [c_void_p, _PF, _PF, c_int64, _PF, c_int64, c_void_p,
                                                        c_int64, _PF, c_int32, c_void_p, c_int64, c_int64, c_int64,
                                                        _P64, _P64, _P64, _P64, _P64, c_int64, _P64, c_int64]),
    "b2_hmm_smoother": (c_int32, [c_void_p, _PF, c_int64, c_int32, _P64, c_int64, c_void_p, _PF, c_int64, _PF,
                                  c_int64, _PF, c_int64, c_int32, c_int64, c_void_p, c_int64, c_int32, c_int64,
                                  c_int64, c_int64, _PF, _PF, _PF, _PF, _PF, _PF]),
    "b2_hmm_smoother_from_filtered": (c_int32, [c_void_p, _PF, c_int64, _PF, c_int64, c_int32, c_int64, c_void_p,
                                                c_int64, c_int32, c_int64, c_int64, c_int64, _PF, _PF, _PF]),
    "b2_expected_state": (c_int32, [c_void_p, _PF, c_int64, _PF, c_int64, c_void_p, c_int64, _PF, c_int64, c_int64,
                                    _P64, _P64, _P64, _P64, _P64, c_int64, _P64]),
    "b2_multiaction_probabilities": (c_int32, [c_void_p, _PF, c_void_p, c_void_p, c_int64, c_int32, c_int64,
                                               c_int64, c_int64, c_int64, _P64, _PF]),
    "b2_sequence_infer": (c_int32, [c_void_p, c_int32, _PF, c_int64, c_int32, _P64, c_int64, c_void_p, _PF, c_int64,
                                    _PF, c_int64, _PF, c_int64, _PF, c_int64, c_int64, c_int64, c_int64, _P64, _P64,
                                    c_int64, _P64, _P64, c_int64, _P64, c_int32, ctypes.c_float]),
    "b2_rollout_setup": (c_int32, [c_void_p, c_void_p, c_int64, c_void_p, c_int32]),
    "b2_rollout": (c_int32, [c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_uint64, c_int32,
                             c_int32, c_void_p]),
}

# ------------------------------------------------ uneven-size rollout structs
RO_MAX_F, RO_MAX_M, RO_MAX_S, RO_MAX_O = 4, 8, 64, 32
RO_MAX_K, RO_MAX_STOT, RO_MAX_P, RO_MAX_COLS, RO_TAB_FLOATS = 4096, 256, 1024, 64, 6144


class RoAgent(ctypes.Structure):
    """``b2_ro_agent``."""

    _fields_ = [("F", c_int32), ("M", c_int32), ("T", c_int32), ("P", c_int32), ("n_multi", c_int32),
                ("w0", c_int32), ("S_tot", c_int32), ("sum_K", c_int32), ("S", c_int32 * RO_MAX_F),
                ("U", c_int32 * RO_MAX_F), ("qs_off", c_int32 * RO_MAX_F), ("ustride", c_int32 * RO_MAX_F),
                ("obs_mask", c_int32), ("n_multi_r", c_int32), ("P_r", c_int32), ("w0_r", c_int32),
                ("ustride_r", c_int32 * RO_MAX_F), ("O", c_int32 * RO_MAX_M), ("K", c_int32 * RO_MAX_M), ("rank", c_int32 * RO_MAX_M),
                ("dep", (c_int32 * RO_MAX_F) * RO_MAX_M), ("dstride", (c_int32 * RO_MAX_F) * RO_MAX_M),
                ("A_off", c_int64 * RO_MAX_M), ("C_off", c_int64 * RO_MAX_M), ("B_off", c_int64 * RO_MAX_F),
                ("D_off", c_int64), ("ll_off", c_int64), ("qs_base", c_int64), ("G_off", c_int64),
                ("gamma", c_float), ("reserved", c_int32)]


class RoTile(ctypes.Structure):
    """``b2_ro_tile``."""

    _fields_ = [("agent", c_int32), ("p_lo", c_int32), ("p_hi", c_int32), ("reserved", c_int32)]


class RoBuffers(ctypes.Structure):
    """``b2_ro_buffers`` (device addresses)."""

    _fields_ = [("agents", c_void_p), ("tiles", c_void_p), ("Aprime", c_void_p), ("Aprime_bf16", c_void_p),
                ("Aprime_count", c_int64), ("B", c_void_p), ("B_count", c_int64), ("C", c_void_p),
                ("C_count", c_int64), ("D", c_void_p), ("D_count", c_int64), ("ll", c_void_p), ("ll_count", c_int64),
                ("qs", c_void_p), ("qs64", c_void_p), ("qs_count", c_int64), ("G", c_void_p), ("G_count", c_int64),
                ("env_state", c_void_p), ("obs", c_void_p), ("rec_obs", c_void_p), ("rec_state", c_void_p),
                ("rec_action", c_void_p), ("rec_qs", c_void_p), ("rec_G", c_void_p), ("sync", c_void_p),
                ("sync_count", c_int64)]


class RoConfig(ctypes.Structure):
    """``b2_ro_config``."""

    _fields_ = [("threads", c_int32), ("kc", c_int32), ("cols", c_int32), ("precision", c_int32)]

_lib = None
_load_error: Exception | None = None


def load():
    """Load and type the library (idempotent). Raises if unavailable."""
    global _lib, _load_error
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"pymdp_b200 native library not found at {LIB_PATH}; "
                           "build it with `python -m pymdp_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def is_available() -> bool:
    """True if the native library loads (mirrors ``pymdp.ffi.is_available``)."""
    try:
        load()
        return True
    except Exception as exc:  # noqa: BLE001
        global _load_error
        _load_error = exc
        return False


def last_error() -> str:
    return load().b2_last_error().decode()


def check(rc: int) -> None:
    if rc == B2_OK:
        return
    msg = last_error()
    if rc == B2_ERR_INVALID_ARGUMENT:
        raise InvalidArgumentError(rc, msg)
    if rc == B2_ERR_UNSUPPORTED:
        raise UnsupportedError(rc, msg)
    raise B2Error(rc, msg)


def i64(values) -> ctypes.Array:
    """Host int64 attribute array (kept alive by the caller)."""
    vals = [int(v) for v in values]
    arr = (c_int64 * max(1, len(vals)))(*vals)
    return arr


def launch_count() -> int:
    return int(load().b2_launch_count())
