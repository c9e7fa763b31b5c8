"""Drop-in host mirror of the reference's ``pymdp.ffi`` for the FPI and EFE paths.

Same names, argument meaning, batching convention and error behaviour as
``pymdp/ffi/_fpi.py`` and ``pymdp/ffi/_efe.py``; arrays are torch CUDA
tensors (device memory is the only thing torch is used for here). Every
call goes through the C-ABI in ``include/pymdp_b200.h`` on the current torch
stream and never synchronises.

Batching follows ``jax.ffi.ffi_call(..., vmap_method="broadcast_all")``: an
optional leading batch axis on every per-agent input; the kernel iterates
over the batch internally (one launch per call).
"""

from __future__ import annotations

import ctypes

from typing import Sequence

import numpy as np
import torch

from . import _lib
from ._lib import (FLAG_FACTORED, FLAG_MODEL_PARAMS_STATIC, FLAG_POLICY_TREE, FLAG_USE_INDUCTIVE, FLAG_USE_PARAM_INFO_GAIN,  # noqa: F401
                   FLAG_USE_STATES_INFO_GAIN, FLAG_USE_UTILITY, MAX_DEP_RANK, PRECISIONS, PRECISION_SHIFT,
                   B2Error, InvalidArgumentError, UnsupportedError, check, i64, is_available)

MAX_FFI_DEP_RANK = MAX_DEP_RANK

__all__ = [
    "MAX_FFI_DEP_RANK", "FLAG_USE_UTILITY", "FLAG_USE_STATES_INFO_GAIN", "FLAG_USE_INDUCTIVE",
    "FLAG_USE_PARAM_INFO_GAIN", "FLAG_MODEL_PARAMS_STATIC", "is_available", "can_handle_fpi", "fpi_ffi",
    "fpi_obs", "can_handle", "neg_efe_all_policies_ffi", "policy_posterior", "select_action",
    "flatten_ragged_f32", "flatten_dep_lists", "dep_list_rank_ok", "dep_indices_in_range", "B2Error",
]


# ------------------------------------------------------------------ helpers
def dep_list_rank_ok(deps: Sequence[int]) -> bool:
    """``pymdp/ffi/_core.py:83-86``."""
    return 1 <= len(deps) <= MAX_FFI_DEP_RANK


def dep_indices_in_range(deps: Sequence[int], num_factors: int) -> bool:
    """``pymdp/ffi/_core.py:89-91``."""
    return all(0 <= d < num_factors for d in deps)


def flatten_dep_lists(dep_lists: Sequence[Sequence[int]]) -> tuple[np.ndarray, np.ndarray]:
    """``pymdp/ffi/_core.py:267-279``: ``(flat_int64, offsets_int64)``."""
    offsets = np.zeros(len(dep_lists) + 1, dtype=np.int64)
    for i, deps in enumerate(dep_lists):
        offsets[i + 1] = offsets[i] + len(deps)
    flat = np.array([d for deps in dep_lists for d in deps], dtype=np.int64)
    return flat, offsets


def _stream(t: torch.Tensor):
    return torch.cuda.current_stream(t.device).cuda_stream


def _dev_f32(x, device=None) -> torch.Tensor:
    if not isinstance(x, torch.Tensor):
        x = torch.as_tensor(np.asarray(x, dtype=np.float32))
    if device is not None and x.device != device:
        x = x.to(device)
    if x.dtype != torch.float32:
        x = x.float()
    return x


def _require_cuda(t: torch.Tensor, what: str) -> None:
    if t.device.type != "cuda":
        raise ValueError(f"{what} must be a CUDA tensor (this library has no CPU path)")


def flatten_ragged_f32(arrays: Sequence[torch.Tensor], batch_ndim: int = 0,
                       device=None) -> tuple[torch.Tensor, np.ndarray]:
    """``pymdp/ffi/_core.py:247-264`` with an optional leading batch axis.

    Returns ``(flat, offsets)``: ``flat`` is ``[*batch, sum_i size_i]``
    float32 (contiguous), ``offsets`` the int64 prefix sums of the
    per-array (per-agent) sizes.
    """
    arrays = [_dev_f32(a, device) for a in arrays]
    lead = tuple(arrays[0].shape[:batch_ndim]) if arrays else ()
    chunks = [a.reshape(lead + (int(np.prod(a.shape[batch_ndim:])),)) for a in arrays]
    offsets = np.zeros(len(chunks) + 1, dtype=np.int64)
    for i, c in enumerate(chunks):
        offsets[i + 1] = offsets[i] + c.shape[-1]
    flat = torch.cat(chunks, dim=-1).contiguous() if chunks else torch.zeros(0)
    return flat, offsets


# ---------------------------------------------------------------------- FPI
def can_handle_fpi(prior: Sequence, A_dependencies: Sequence[Sequence[int]], num_iter: int) -> bool:
    """``pymdp/ffi/_fpi.py:22-65``: the FPI kernel can run this problem.

    Same restrictions (num_iter > 0, F >= 1, M >= 1, ranks in [1, 8], indices
    in range, distinct factors per modality, library loadable) plus this
    build's F <= 16, M <= 32 limits.
    """
    if not is_available() or num_iter <= 0:
        return False
    F, M = len(prior), len(A_dependencies)
    if F < 1 or M < 1 or F > _lib.MAX_FACTORS or M > _lib.MAX_MODALITIES:
        return False
    for deps in A_dependencies:
        if not dep_list_rank_ok(deps) or not dep_indices_in_range(deps, F) or len(set(deps)) != len(deps):
            return False
    return True


def _validate_fpi_inputs(log_likelihoods, log_prior, A_dependencies, num_iter):
    """``pymdp/ffi/_fpi.py:95-140``."""
    F, M = len(log_prior), len(log_likelihoods)
    if F < 1 or M < 1:
        raise ValueError("FPI FFI requires at least one factor and one modality")
    if not can_handle_fpi(log_prior, A_dependencies, num_iter):
        raise ValueError("FPI FFI cannot handle this problem (rank > 8, num_iter <= 0, or library unavailable)")
    if len(A_dependencies) != M:
        raise ValueError(f"A_dependencies length {len(A_dependencies)} does not match len(log_likelihoods) = {M}")
    S = [int(np.shape(lp)[-1]) for lp in log_prior]
    for m, (ll, deps) in enumerate(zip(log_likelihoods, A_dependencies)):
        shp = tuple(np.shape(ll))
        if len(shp) < len(deps):
            raise ValueError(f"log_likelihoods[{m}] rank {len(shp)} < |A_deps[{m}]| = {len(deps)}")
        trailing = shp[len(shp) - len(deps):]
        expected = tuple(S[d] for d in deps)
        if trailing != expected:
            raise ValueError(f"log_likelihoods[{m}] trailing shape {trailing} does not match expected "
                             f"{expected} from A_dependencies[{m}] = {tuple(deps)}")
    return S


def fpi_ffi(log_likelihoods: Sequence[torch.Tensor], log_prior: Sequence[torch.Tensor],
            A_dependencies: Sequence[Sequence[int]], num_iter: int) -> list[torch.Tensor]:
    """``pymdp/ffi/_fpi.py:143-270``: posterior marginals from ll and log prior.

    ``log_likelihoods[m]`` has shape ``(*batch, *S[A_dependencies[m]])`` and
    ``log_prior[f]`` shape ``(*batch, S_f)``; returns ``qs[f]`` of shape
    ``(*batch, S_f)``. Exactly ``num_iter`` iterations (reference JAX
    semantics). One kernel launch.
    """
    S = _validate_fpi_inputs(log_likelihoods, log_prior, A_dependencies, num_iter)
    F = len(S)
    dev = log_prior[0].device if isinstance(log_prior[0], torch.Tensor) else torch.device("cuda")
    lead = tuple(np.shape(log_prior[0])[:-1])
    nb = len(lead)
    ll_flat, ll_offsets = flatten_ragged_f32(
        [torch.broadcast_to(_dev_f32(l, dev), lead + tuple(np.shape(l)[-len(d):]))
         for l, d in zip(log_likelihoods, A_dependencies)], nb, dev)
    lp_flat, lp_offsets = flatten_ragged_f32(
        [torch.broadcast_to(_dev_f32(l, dev), lead + (S[f],)) for f, l in enumerate(log_prior)], nb, dev)
    _require_cuda(lp_flat, "log_prior")
    q = torch.empty_like(lp_flat)
    _require_cuda(ll_flat, "log_likelihoods")
    dep_flat, dep_offs = flatten_dep_lists(A_dependencies)
    attrs = [i64(S), i64(ll_offsets), i64(lp_offsets), i64(dep_flat), i64(dep_offs)]
    check(_lib.load().b2_fpi(_stream(q), ll_flat.data_ptr(), ll_flat.numel(), lp_flat.data_ptr(), lp_flat.numel(),
                             q.data_ptr(), q.numel(), attrs[0], F, attrs[1], len(ll_offsets), attrs[2],
                             len(lp_offsets), attrs[3], len(dep_flat), attrs[4], len(dep_offs), int(num_iter)))
    return [q[..., int(lp_offsets[f]):int(lp_offsets[f + 1])] for f in range(F)]


def fpi_obs_flat(A_flat: torch.Tensor, A_agent_stride: int, A_offsets, O, obs: torch.Tensor,
                 prior_flat: torch.Tensor, S, A_dependencies, num_iter: int,
                 out: torch.Tensor | None = None) -> torch.Tensor:
    """Fused-observation FPI on pre-flattened device buffers (no copies).

    ``A_flat``: agent b's A at ``b * A_agent_stride`` (0 = shared);
    ``obs``: ``[batch, M]`` int32; ``prior_flat``: ``[batch, sum S]``.
    Returns / fills ``q`` of shape ``[batch, sum S]``.
    """
    batch = obs.shape[0]
    q = out if out is not None else torch.empty_like(prior_flat)
    for t, what in ((A_flat, "A"), (obs, "obs"), (prior_flat, "prior"), (q, "out")):
        _require_cuda(t, what)
    if obs.dtype != torch.int32 or not obs.is_contiguous():
        raise ValueError("obs must be a contiguous int32 tensor")
    dep_flat, dep_offs = flatten_dep_lists(A_dependencies)
    attrs = [i64(A_offsets), i64(O), i64(S), i64(dep_flat), i64(dep_offs)]
    check(_lib.load().b2_fpi_obs(_stream(q), A_flat.data_ptr(), int(A_agent_stride), attrs[0], len(A_offsets),
                                 attrs[1], len(O), obs.data_ptr(), prior_flat.data_ptr(), q.data_ptr(), batch,
                                 attrs[2], len(S), attrs[3], len(dep_flat), attrs[4], len(dep_offs),
                                 int(num_iter)))
    return q


def fpi_obs(A: Sequence[torch.Tensor], obs, prior: Sequence[torch.Tensor],
            A_dependencies: Sequence[Sequence[int]], num_iter: int) -> list[torch.Tensor]:
    """``algos.run_factorized_fpi`` with one-hot observations, fully fused.

    ``A[m]``: ``(batch, O_m, *S_deps)`` per agent or ``(O_m, *S_deps)`` shared;
    ``obs``: ``(batch, M)`` observation indices; ``prior[f]``: ``(batch, S_f)``.
    The observed log-A slices and the log prior are formed in-kernel.
    """
    if not can_handle_fpi(prior, A_dependencies, num_iter):
        raise ValueError("FPI cannot handle this problem (rank > 8, num_iter <= 0, duplicate deps, limits)")
    dev = prior[0].device
    S = [int(p.shape[-1]) for p in prior]
    batch = int(prior[0].shape[0])
    shared = A[0].ndim == len(A_dependencies[0]) + 1
    O = [int(a.shape[0] if shared else a.shape[1]) for a in A]
    A_flat, A_offsets = flatten_ragged_f32(A, 0 if shared else 1, dev)
    prior_flat, _ = flatten_ragged_f32(prior, 1, dev)
    obs_t = torch.as_tensor(obs, device=dev).to(torch.int32).contiguous()
    if obs_t.shape != (batch, len(A)):
        raise ValueError(f"obs must have shape {(batch, len(A))}, got {tuple(obs_t.shape)}")
    q = fpi_obs_flat(A_flat, 0 if shared else int(A_offsets[-1]), A_offsets, O, obs_t, prior_flat, S,
                     A_dependencies, num_iter)
    offs = np.cumsum([0] + S)
    return [q[:, offs[f]:offs[f + 1]] for f in range(len(S))]


# ---------------------------------------------------------------------- EFE
def can_handle(A_dependencies, B_dependencies, use_param_info_gain: bool, *, num_factors: int | None = None,
               num_modalities: int | None = None, ffi_beneficial: bool | None = None,
               use_inductive: bool = False) -> bool:
    """``pymdp/ffi/_efe.py:296-358``: the EFE kernel can run this problem.

    ``ffi_beneficial`` is accepted for signature parity (the reference's
    Orin roofline router); this build always prefers the GPU path. The
    parameter-information-gain and inductive terms are computed by the FP32
    SIMT kernel whatever precision is requested.
    """
    if not is_available():
        return False
    if num_modalities is not None and len(A_dependencies) != num_modalities:
        return False
    if num_factors is not None and len(B_dependencies) != num_factors:
        return False
    if len(A_dependencies) > _lib.MAX_MODALITIES or len(B_dependencies) > _lib.MAX_FACTORS:
        return False
    for deps in list(A_dependencies) + list(B_dependencies):
        if not dep_list_rank_ok(deps):
            return False
        if num_factors is not None and not dep_indices_in_range(deps, num_factors):
            return False
    return True


def efe_flags(use_utility=True, use_states_info_gain=True, use_param_info_gain=False, use_inductive=False,
              ffi_cache_params_static=False, precision="fp32", policy_tree=False, factored=False) -> int:
    """Flag word of ``b2_neg_efe``. ``policy_tree`` declares the policy matrix
    to be ``construct_policies``' full product set (``B2_FLAG_POLICY_TREE``):
    the tensor-core paths then evaluate each distinct prefix once. With it,
    ``factored`` (``B2_FLAG_FACTORED``) contracts A factor by factor over the
    distinct per-factor marginals when the transitions are factor-local."""
    flags = FLAG_POLICY_TREE if policy_tree else 0
    flags |= FLAG_FACTORED if (factored and policy_tree) else 0
    flags |= FLAG_USE_UTILITY if use_utility else 0
    flags |= FLAG_USE_STATES_INFO_GAIN if use_states_info_gain else 0
    flags |= FLAG_USE_INDUCTIVE if use_inductive else 0
    flags |= FLAG_USE_PARAM_INFO_GAIN if use_param_info_gain else 0
    flags |= FLAG_MODEL_PARAMS_STATIC if ffi_cache_params_static else 0
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    return flags | (PRECISIONS[precision] << PRECISION_SHIFT)


class EfeLayout:
    """Host attribute arrays of one model structure (the 13 int64 spans)."""

    def __init__(self, S, O, U, T, A_dependencies, B_dependencies, I_depths=None):
        F, M = len(S), len(O)
        self.S, self.O, self.U, self.T = [int(s) for s in S], [int(o) for o in O], [int(u) for u in U], int(T)
        self.F, self.M = F, M
        self.A_dependencies = [list(map(int, d)) for d in A_dependencies]
        self.B_dependencies = [list(map(int, d)) for d in B_dependencies]
        self.qs_offsets = np.cumsum([0] + self.S).astype(np.int64)
        KA = [int(np.prod([S[d] for d in deps])) for deps in A_dependencies]
        KB = [int(np.prod([S[d] for d in deps])) for deps in B_dependencies]
        self.A_offsets = np.cumsum([0] + [o * k for o, k in zip(self.O, KA)]).astype(np.int64)
        self.B_offsets = np.cumsum([0] + [s * k * u for s, k, u in zip(self.S, KB, self.U)]).astype(np.int64)
        self.C_offsets = np.cumsum([0] + [self.T * o for o in self.O]).astype(np.int64)
        self.I_depths = np.array(I_depths if I_depths is not None else [1] * F, dtype=np.int64)
        self.I_offsets = np.cumsum([0] + [int(d) * s for d, s in zip(self.I_depths, self.S)]).astype(np.int64)
        self.A_dep_flat, self.A_dep_offsets = flatten_dep_lists(self.A_dependencies)
        self.B_dep_flat, self.B_dep_offsets = flatten_dep_lists(self.B_dependencies)
        self._c = [i64(x) for x in (self.S, self.O, self.U, self.qs_offsets, self.A_offsets, self.B_offsets,
                                    self.C_offsets, self.I_offsets, self.I_depths, self.A_dep_flat,
                                    self.A_dep_offsets, self.B_dep_flat, self.B_dep_offsets)]

    def pack_bytes(self, Bn: int, P: int, flags: int) -> int:
        """Bytes of the tensor-core pack cache (``b2_neg_efe_pack_bytes``)."""
        c = self._c
        n = ctypes.c_int64(0)
        check(_lib.load().b2_neg_efe_pack_bytes(
            int(Bn), int(P), self.T, self.F, self.M, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[9],
            len(self.A_dep_flat), c[10], c[11], len(self.B_dep_flat), c[12], int(flags), ctypes.byref(n)))
        return int(n.value)

    def call(self, stream, pm, pm_batched, qs, A, B, C, I, pA, pB, eps, out, Bn, P, flags, cache=None):
        """``b2_neg_efe``; with ``cache = (uint8 device tensor, ctypes.c_int32
        valid flag)`` the tensor-core operand images are packed once and
        reused (``b2_neg_efe_cached``)."""
        c = self._c
        for t in (pm, qs, A, B, C, I, pA, pB, eps, out):
            if t is not None:
                _require_cuda(t, "neg-EFE buffer")
        if stream is None:
            stream = _stream(out)
        ptr = (lambda t: 0 if t is None else t.data_ptr())
        cnt = (lambda t: 0 if t is None else t.numel())
        args = (stream, ptr(pm), cnt(pm), int(pm_batched), ptr(qs), cnt(qs), ptr(A), cnt(A), ptr(B), cnt(B), ptr(C),
                cnt(C), ptr(I), cnt(I), ptr(pA), cnt(pA), ptr(pB), cnt(pB), ptr(eps), cnt(eps), ptr(out), cnt(out),
                int(Bn), int(P), self.T, self.F, self.M, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[9],
                len(self.A_dep_flat), c[10], c[11], len(self.B_dep_flat), c[12], int(flags))
        if cache is None:
            check(_lib.load().b2_neg_efe(*args))
        else:
            buf, valid = cache
            _require_cuda(buf, "pack cache")
            check(_lib.load().b2_neg_efe_cached(*args, buf.data_ptr(), buf.numel(), ctypes.byref(valid)))

    def learn_A(self, pA: torch.Tensor, A: torch.Tensor, obs: torch.Tensor, qs: torch.Tensor, lr: torch.Tensor,
                Bn: int, T: int, modality_mask: int | None = None, categorical: bool = False):
        """``b2_update_obs_likelihood_dirichlet`` in place on the flattened
        ``pA`` / ``A`` ([Bn, A_offsets[M]]): ``obs`` int32 [Bn, T, M] (or float
        [Bn, T, sum O] when ``categorical``), ``qs`` [Bn, T, S_tot], ``lr`` [Bn]
        or one value (device)."""
        for t in (pA, A, obs, qs, lr):
            _require_cuda(t, "learning buffer")
        c = self._c
        mask = (1 << self.M) - 1 if modality_mask is None else int(modality_mask)
        check(_lib.load().b2_update_obs_likelihood_dirichlet(
            _stream(pA), pA.data_ptr(), A.data_ptr(), A.numel(), 0 if categorical else obs.data_ptr(),
            obs.data_ptr() if categorical else 0, obs.numel(), qs.data_ptr(), qs.numel(), lr.data_ptr(),
            int(lr.numel() != 1), int(Bn), int(T), self.F, self.M, c[0], c[1], c[3], c[4], c[9], len(self.A_dep_flat),
            c[10], mask))

    def learn_B(self, pB: torch.Tensor, B: torch.Tensor, qs: torch.Tensor, actions: torch.Tensor, lr: torch.Tensor,
                workspace: torch.Tensor, Bn: int, T: int, factor_mask: int | None = None):
        """``b2_update_state_transition_dirichlet`` in place on the flattened
        ``pB`` / ``B`` ([Bn, B_offsets[F]]): ``qs`` [Bn, T, S_tot] belief
        sequence, ``actions`` int32 [Bn, T-1, F], ``workspace`` one device int32."""
        for t in (pB, B, qs, actions, lr, workspace):
            _require_cuda(t, "learning buffer")
        c = self._c
        mask = (1 << self.F) - 1 if factor_mask is None else int(factor_mask)
        check(_lib.load().b2_update_state_transition_dirichlet(
            _stream(pB), pB.data_ptr(), B.data_ptr(), B.numel(), qs.data_ptr(), qs.numel(), actions.data_ptr(),
            actions.numel(), lr.data_ptr(), int(lr.numel() != 1), workspace.data_ptr(), int(Bn), int(T), self.F,
            c[0], c[2], c[3], c[5], c[11], len(self.B_dep_flat), c[12], mask))


    def learn_B_joint(self, pB: torch.Tensor, B: torch.Tensor, joint: torch.Tensor, actions: torch.Tensor,
                      lr: torch.Tensor, workspace: torch.Tensor, Bn: int, T: int, factor_mask: int | None = None):
        """``b2_update_state_transition_from_joint`` in place on the flattened
        ``pB`` / ``B``: ``joint`` ``[Bn, sum_f (T-1) S_f K_f]`` (per factor the
        ``(T-1, S_f, *S_deps)`` pairwise posteriors), ``actions`` int32
        ``[Bn, T-1, F]``, ``workspace`` one device int32."""
        for t in (pB, B, joint, actions, lr, workspace):
            _require_cuda(t, "learning buffer")
        c = self._c
        mask = (1 << self.F) - 1 if factor_mask is None else int(factor_mask)
        check(_lib.load().b2_update_state_transition_from_joint(
            _stream(pB), pB.data_ptr(), B.data_ptr(), B.numel(), joint.data_ptr(), joint.numel(), actions.data_ptr(),
            actions.numel(), lr.data_ptr(), int(lr.numel() != 1), workspace.data_ptr(), int(Bn), int(T), self.F,
            c[0], c[2], c[3], c[5], c[11], len(self.B_dep_flat), c[12], mask))



def neg_efe_all_policies_ffi(policy_matrix, qs_init, A, B, C, I, A_dependencies, B_dependencies, *,
                             pA=None, pB=None, use_utility: bool = True, use_states_info_gain: bool = True,
                             use_param_info_gain: bool = False, use_inductive: bool = True,
                             inductive_epsilon: float = 1e-3, ffi_cache_params_static: bool = False,
                             precision: str = "fp32", policy_tree: bool = False,
                             factored: bool = False) -> torch.Tensor:
    """``pymdp/ffi/_efe.py:491-711``: ``neg_efe`` (G) of every policy.

    ``qs_init[f]``: ``(*batch, S_f)``; ``A[m]``: ``(*batch, O_m, *S_deps)``;
    ``B[f]``: ``(*batch, S_f, *S_Bdeps, U_f)``; ``C[m]``: ``(*batch, O_m)`` or
    ``(*batch, T, O_m)``; ``I[f]``: ``(*batch, depth_f, S_f)``;
    ``policy_matrix``: ``(P, T, F)`` int. Returns ``(*batch, P)``.
    Caller applies gamma + softmax + log E (see :func:`policy_posterior`).
    """
    if use_param_info_gain and not pA and not pB:
        raise ValueError("use_param_info_gain=True requires at least one of pA, pB")
    F, M = len(qs_init), len(A)
    if F < 1 or M < 1:
        raise ValueError("neg-EFE FFI requires at least one factor and one modality")
    if len(B) != F or len(I) != F:
        raise ValueError("B and I must have one entry per hidden-state factor")
    if len(C) != M:
        raise ValueError("C must have one entry per observation modality")
    if not can_handle(A_dependencies, B_dependencies, use_param_info_gain, num_factors=F, num_modalities=M,
                      use_inductive=use_inductive):
        raise ValueError("unsupported or inconsistent A/B dependency metadata")
    dev = qs_init[0].device if isinstance(qs_init[0], torch.Tensor) else torch.device("cuda")
    pm = torch.as_tensor(policy_matrix, device=dev).to(torch.int32).contiguous()
    if pm.ndim != 3:
        raise ValueError(f"policy_matrix must have shape (P, T, F); got {tuple(pm.shape)}")
    P, T, Fp = pm.shape
    if P <= 0 or T <= 0 or Fp != F:
        raise ValueError(f"policy_matrix shape {tuple(pm.shape)} is inconsistent with {F} factors")
    lead = tuple(np.shape(qs_init[0])[:-1])
    nb = len(lead)
    Bn = int(np.prod(lead)) if nb else 1
    S = [int(np.shape(q)[-1]) for q in qs_init]
    O = [int(np.shape(a)[nb]) for a in A]
    U = [int(np.shape(b)[-1]) for b in B]
    for m, (a, deps) in enumerate(zip(A, A_dependencies)):
        exp = lead + (O[m],) + tuple(S[d] for d in deps)
        if tuple(np.shape(a)) != exp:
            raise ValueError(f"A[{m}] shape {tuple(np.shape(a))} does not match expected {exp}")
    for f, (b, deps) in enumerate(zip(B, B_dependencies)):
        exp = lead + (S[f],) + tuple(S[d] for d in deps) + (U[f],)
        if tuple(np.shape(b)) != exp:
            raise ValueError(f"B[{f}] shape {tuple(np.shape(b))} does not match expected {exp}")
    C_t = []
    for m, c in enumerate(C):
        c = _dev_f32(c, dev)
        shp = tuple(c.shape[nb:])
        if shp == (O[m],):
            c = c.unsqueeze(-2).expand(lead + (T, O[m]))
        elif shp != (T, O[m]):
            raise ValueError(f"C[{m}] must have shape (O_m,) or (T, O_m); got {shp}")
        C_t.append(c)
    I_depths = [int(np.shape(i)[-2]) for i in I]
    lay = EfeLayout(S, O, U, T, A_dependencies, B_dependencies, I_depths)
    qs_flat, _ = flatten_ragged_f32(qs_init, nb, dev)
    A_flat, _ = flatten_ragged_f32(A, nb, dev)
    B_flat, _ = flatten_ragged_f32(B, nb, dev)
    C_flat, _ = flatten_ragged_f32(C_t, nb, dev)
    I_flat, _ = flatten_ragged_f32(I, nb, dev)
    _require_cuda(A_flat, "A")
    pA_flat = pB_flat = None
    if use_param_info_gain and pA:
        for m, (pa, a) in enumerate(zip(pA, A)):
            if tuple(np.shape(pa)) != tuple(np.shape(a)):
                raise ValueError(f"pA[{m}] shape {tuple(np.shape(pa))} does not match A[{m}] {tuple(np.shape(a))}")
        pA_flat, _ = flatten_ragged_f32(pA, nb, dev)
    if use_param_info_gain and pB:
        for f, (pb, bb) in enumerate(zip(pB, B)):
            if tuple(np.shape(pb)) != tuple(np.shape(bb)):
                raise ValueError(f"pB[{f}] shape {tuple(np.shape(pb))} does not match B[{f}] {tuple(np.shape(bb))}")
        pB_flat, _ = flatten_ragged_f32(pB, nb, dev)
    eps = _dev_f32(torch.as_tensor(inductive_epsilon, dtype=torch.float32), dev).reshape(-1).contiguous()
    out = torch.empty(lead + (P,), dtype=torch.float32, device=dev)
    flags = efe_flags(use_utility, use_states_info_gain, use_param_info_gain, use_inductive,
                      ffi_cache_params_static, precision, policy_tree=policy_tree, factored=factored)
    lay.call(None, pm, 0, qs_flat, A_flat, B_flat, C_flat, I_flat, pA_flat, pB_flat, eps, out, Bn, P, flags)
    return out


def policy_posterior(neg_efe: torch.Tensor, E: torch.Tensor, gamma) -> torch.Tensor:
    """``q_pi = softmax(gamma * neg_efe + log_stable(E))`` (``control.py:349``)."""
    neg_efe = neg_efe.contiguous()
    dev = neg_efe.device
    P = neg_efe.shape[-1]
    Bn = neg_efe.numel() // P
    E = _dev_f32(E, dev).contiguous()
    g = _dev_f32(torch.as_tensor(gamma, dtype=torch.float32), dev).reshape(-1).contiguous()
    q = torch.empty_like(neg_efe)
    for t in (neg_efe, E, g):
        _require_cuda(t, "policy_posterior buffer")
    check(_lib.load().b2_policy_posterior(_stream(q), neg_efe.data_ptr(), E.data_ptr(), int(E.numel() != P),
                                          g.data_ptr(), int(g.numel() != 1), q.data_ptr(), Bn, P))
    return q


def sample_action(q_pi: torch.Tensor, policy_matrix, num_controls, sampling_mode: str = "full",
                  action_selection: str = "deterministic", alpha=16.0, seed: int | None = None):
    """``Agent.sample_action`` (``pymdp/agent.py:939-967``): ``sampling_mode``
    "full" (``control.sample_policy``) or "marginal" (``control.sample_action``
    over ``get_marginals``), ``action_selection`` "deterministic" or
    "stochastic" (needs ``seed``: a counter-based generator stands in for
    JAX's key). Returns ``(batch, F)`` int32."""
    if sampling_mode not in ("full", "marginal"):
        raise ValueError("sampling_mode must be 'full' or 'marginal'")
    if action_selection not in ("deterministic", "stochastic"):
        raise ValueError("action_selection must be 'deterministic' or 'stochastic'")
    if action_selection == "stochastic" and seed is None:
        raise ValueError("Please provide a random number generator key to sample actions stochastically")
    q_pi = q_pi.contiguous()
    pm = torch.as_tensor(policy_matrix, device=q_pi.device).to(torch.int32).contiguous()
    P, T, F = pm.shape
    Bn = q_pi.numel() // P
    act = torch.empty(q_pi.shape[:-1] + (F,), dtype=torch.int32, device=q_pi.device)
    _require_cuda(q_pi, "q_pi")
    a = _dev_f32(torch.as_tensor(alpha, dtype=torch.float32), q_pi.device).reshape(-1).contiguous()
    check(_lib.load().b2_sample_action(_stream(act), q_pi.data_ptr(), pm.data_ptr(), i64(list(num_controls)),
                                       act.data_ptr(), Bn, P, T, F, int(sampling_mode == "marginal"),
                                       int(action_selection == "stochastic"), a.data_ptr(), int(a.numel() != 1),
                                       int(seed or 0) & ((1 << 64) - 1)))
    return act


def select_action(q_pi: torch.Tensor, policy_matrix: torch.Tensor) -> torch.Tensor:
    """Deterministic ``sample_policy`` (``control.py:115-150``): ``(batch, F)`` int32."""
    q_pi = q_pi.contiguous()
    pm = torch.as_tensor(policy_matrix, device=q_pi.device).to(torch.int32).contiguous()
    P, T, F = pm.shape
    Bn = q_pi.numel() // P
    act = torch.empty(q_pi.shape[:-1] + (F,), dtype=torch.int32, device=q_pi.device)
    _require_cuda(q_pi, "q_pi")
    check(_lib.load().b2_select_action(_stream(act), q_pi.data_ptr(), pm.data_ptr(), act.data_ptr(), Bn, P, T, F))
    return act


def expected_state(qs_flat: torch.Tensor, B_flat: torch.Tensor, action: torch.Tensor, lay: "EfeLayout",
                   out: torch.Tensor | None = None) -> torch.Tensor:
    """``b2_expected_state``: ``compute_expected_state`` (``pymdp/control.py:
    351-389``) per agent on flattened beliefs ``[Bn, sum S]`` and transitions
    ``[Bn, B_offsets[F]]`` with ``action`` int32 ``[Bn, F]``."""
    for t in (qs_flat, B_flat, action):
        _require_cuda(t, "expected-state buffer")
    Bn = qs_flat.shape[0]
    act = action.to(torch.int32).contiguous()
    out = torch.empty_like(qs_flat) if out is None else out
    c = lay._c
    check(_lib.load().b2_expected_state(_stream(out), qs_flat.data_ptr(), qs_flat.numel(), B_flat.data_ptr(),
                                        B_flat.numel(), act.data_ptr(), act.numel(), out.data_ptr(), int(Bn), lay.F,
                                        c[0], c[2], c[3], c[5], c[11], len(lay.B_dep_flat), c[12]))
    return out


def unique_multiactions(policy_matrix, num_controls) -> np.ndarray:
    """The reference's ``Agent.unique_multiactions`` (``pymdp/agent.py:396-399``):
    the sorted distinct first-step joint actions, padded with -1 rows to
    ``prod(num_controls)`` rows (``jnp.unique(..., size=, fill_value=-1)``)."""
    first = np.unique(np.asarray(policy_matrix)[:, 0], axis=0)
    size = int(np.prod(num_controls))
    out = np.full((size, first.shape[1]), -1, dtype=np.int32)
    out[:min(size, len(first))] = first[:size]
    return out


def multiaction_probabilities(q_pi: torch.Tensor, policy_matrix: torch.Tensor, unique: torch.Tensor,
                              num_controls, sampling_mode: str = "full") -> torch.Tensor:
    """``b2_multiaction_probabilities``: ``Agent.multiaction_probabilities``
    (``pymdp/agent.py:908-937``) for a batch ``q_pi [Bn, P]``; returns
    ``[Bn, prod(num_controls)]``."""
    if sampling_mode not in ("full", "marginal"):
        raise ValueError("sampling_mode must be 'full' or 'marginal'")
    _require_cuda(q_pi, "q_pi")
    q_pi = q_pi.contiguous()
    pm = torch.as_tensor(policy_matrix, device=q_pi.device).to(torch.int32).contiguous()
    uq = torch.as_tensor(unique, device=q_pi.device).to(torch.int32).contiguous()
    P, T, F = pm.shape
    Bn = q_pi.numel() // P
    n = int(uq.shape[0])
    out = torch.empty(q_pi.shape[:-1] + (n,), dtype=torch.float32, device=q_pi.device)
    check(_lib.load().b2_multiaction_probabilities(_stream(out), q_pi.data_ptr(), pm.data_ptr(), uq.data_ptr(), n,
                                                   int(sampling_mode == "marginal"), Bn, P, T, F,
                                                   i64(list(num_controls)), out.data_ptr()))
    return out
