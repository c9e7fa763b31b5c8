"""ctypes wrappers over the reference's own CPU FFI kernels (``oracle/_ref``,
built by ``oracle/ref_build.py``): the reference's NegEfeCpu and FpiCpu with
the buffers and attributes its XLA FFI handlers take
(pymdp/ffi/registration/xla_register.cc:118-157, pymdp/ffi/neg_efe/neg_efe.h:60-68,
pymdp/ffi/fpi/fpi.h:18-19).

Test infrastructure: the CPU timing baseline (``bench.py --impl reference``
and ``cpu_baseline``) and a cross-check in ``tests/``. These kernels are FP32
with ``-ffast-math`` and, for FPI, an early stop at max |d log q| < 1e-5
(pymdp/ffi/common/fpi_convergence_tol.h), so they are a timing baseline, not
the parity oracle (the FP64 restatements are).
"""

from __future__ import annotations

import ctypes

import numpy as np

from oracle import ref_build

P_I64 = ctypes.POINTER(ctypes.c_int64)


def _f32(x):
    return np.ascontiguousarray(x, dtype=np.float32)


def _ptr(a, ct=ctypes.c_float):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ct))


def _spans(arrays):
    keep = [np.ascontiguousarray(a, dtype=np.int64) for a in arrays]
    ptrs = (P_I64 * len(keep))(*[k.ctypes.data_as(P_I64) for k in keep])
    lens = (ctypes.c_int64 * len(keep))(*[k.size for k in keep])
    return keep, ptrs, lens


def efe_spans(S, O, U, T, A_deps, B_deps, I_depths=None):
    """The 13 int64 attribute spans of the neg-EFE ABI, in the reference's
    order (S, O, U, qs_offsets, A_offsets, B_offsets, C_offsets, I_offsets,
    I_depths, A_dep_flat, A_dep_offsets, B_dep_flat, B_dep_offsets)."""
    F = len(S)
    KA = [int(np.prod([S[d] for d in dp])) for dp in A_deps]
    KB = [int(np.prod([S[d] for d in dp])) for dp in B_deps]
    I_depths = [1] * F if I_depths is None else list(I_depths)
    cs = lambda xs: np.cumsum([0] + list(xs))  # noqa: E731
    return [np.array(S), np.array(O), np.array(U), cs(S), cs([o * k for o, k in zip(O, KA)]),
            cs([s * k * u for s, k, u in zip(S, KB, U)]), cs([T * o for o in O]),
            cs([d * s for d, s in zip(I_depths, S)]), np.array(I_depths),
            np.array([d for dp in A_deps for d in dp]), cs([len(dp) for dp in A_deps]),
            np.array([d for dp in B_deps for d in dp]), cs([len(dp) for dp in B_deps])]


FLAG_UTILITY, FLAG_INFO_GAIN, FLAG_INDUCTIVE, FLAG_PARAM_INFO_GAIN = 1, 2, 4, 8


def neg_efe_cpu(policies, qs, A, B, C, I, spans, flags=FLAG_UTILITY | FLAG_INFO_GAIN, pA=None, pB=None,
                eps=1e-3) -> np.ndarray:
    """NegEfeCpu over a batch: ``policies`` int32 [Bn, P, T, F] (the
    broadcast_all form) or [P, T, F] (one agent); ``qs``, ``A``, ``B``, ``C``
    (always [T, O_m] per modality), ``I`` ragged-flat float32 [Bn, ...];
    returns neg-EFE [Bn, P] (FP32)."""
    pm = np.ascontiguousarray(policies, dtype=np.int32)
    batched = pm.ndim == 4
    Bn = pm.shape[0] if batched else 1
    P = pm.shape[-3]
    bufs = [_f32(x) for x in (qs, A, B, C, I)]
    pA_, pB_ = (None if x is None else _f32(x) for x in (pA, pB))
    eps_a = np.asarray(eps, dtype=np.float32).reshape(-1 if np.ndim(eps) else ())
    eps_dims = np.array(eps_a.shape, dtype=np.int64)
    out = np.empty((Bn, P), np.float32)
    keep, sp, sl = _spans(spans)
    pm_dims = np.array(pm.shape, dtype=np.int64)
    lib = ref_build.load()
    rc = lib.ref_neg_efe_cpu(
        _ptr(pm, ctypes.c_int32), pm_dims.ctypes.data_as(P_I64), ctypes.c_int32(pm.ndim),
        *[a for b in bufs for a in (_ptr(b), ctypes.c_int64(b.size))],
        _ptr(pA_), ctypes.c_int64(0 if pA_ is None else pA_.size), _ptr(pB_),
        ctypes.c_int64(0 if pB_ is None else pB_.size), _ptr(eps_a), eps_dims.ctypes.data_as(P_I64),
        ctypes.c_int32(eps_a.ndim), _ptr(out), ctypes.c_int64(out.size), sp, sl, ctypes.c_int32(flags))
    del keep
    if rc != 0:
        raise ValueError(lib.ref_last_error().decode())
    return out


def fpi_cpu(ll, lp, S, ll_offsets, A_deps, num_iter=16) -> np.ndarray:
    """FpiCpu: ``ll`` float32 [batch, sum_m K_m] log-likelihoods, ``lp``
    [batch, sum_f S_f] log priors; returns q [batch, sum_f S_f]."""
    ll, lp = _f32(ll), _f32(lp)
    q = np.empty_like(lp)
    spans = [np.array(S), np.asarray(ll_offsets), np.cumsum([0] + list(S)),
             np.array([d for dp in A_deps for d in dp]), np.cumsum([0] + [len(dp) for dp in A_deps])]
    keep, sp, sl = _spans(spans)
    lib = ref_build.load()
    rc = lib.ref_fpi_cpu(_ptr(ll), ctypes.c_int64(ll.size), _ptr(lp), ctypes.c_int64(lp.size), _ptr(q),
                         ctypes.c_int64(q.size), sp, sl, ctypes.c_int32(num_iter))
    del keep
    if rc != 0:
        raise ValueError(lib.ref_last_error().decode())
    return q
