"""Exact single-factor HMM inference over a batch of agents on the GPU.

Mirrors the reference's ``run_exact_single_factor_hmm_scan``
(``pymdp/algos.py:1132-1208``), ``hmm_smoother_from_filtered_colstoch``
(``:1049-1130``) and ``smoothing_exact`` (``pymdp/inference.py:595-634``) with a
leading batch axis on every argument (the reference vmaps them). Each call is
one kernel launch (``b2_hmm_smoother``, ``b2_hmm_smoother_from_filtered``);
transitions follow pymdp's column-stochastic orientation ``B[next, current(, action)]``.
"""

from __future__ import annotations

import torch

from . import _lib
from .ffi import _dev_f32, _require_cuda, _stream, check, i64

_MODES = {"index": 0, "identity": 1}


def _transitions(B0: torch.Tensor, actions, Bn: int, T: int, K: int):
    """(tensor, batched, U, actions int32 or None). With ``actions`` B0 is
    ``(K, K, U)`` or ``(Bn, K, K, U)``. Without: ``(K, K)`` / ``(Bn, K, K)``
    stationary, ``(T-1, K, K)`` / ``(Bn, T-1, K, K)`` time-varying (U = 0), or
    an action axis only when no transition is taken (T = 1) or U = 1."""
    nT = max(T - 1, 0)
    if actions is not None:
        a = torch.as_tensor(actions, device=B0.device)
        if a.ndim == 3 and a.shape[-1] == 1:
            a = a[..., 0]
        a = a.to(torch.int32).reshape(Bn, nT).contiguous()
        if B0.ndim not in (3, 4):
            raise ValueError("with actions, B must be (K, K, U) or (batch, K, K, U)")
        return B0.contiguous(), int(B0.ndim == 4), int(B0.shape[-1]), a
    if B0.ndim == 2:
        return B0.unsqueeze(-1).contiguous(), 0, 1, None
    if B0.ndim == 3:
        if T > 1 and B0.shape[0] == nT and tuple(B0.shape[1:]) == (K, K):
            return B0.contiguous(), 0, 0, None
        if B0.shape[0] == Bn and tuple(B0.shape[1:]) == (K, K):
            return B0.unsqueeze(-1).contiguous(), 1, 1, None
        U = int(B0.shape[-1])
    elif B0.ndim == 4:
        if T > 1 and B0.shape[1] == nT and tuple(B0.shape[2:]) == (K, K):
            return B0.contiguous(), 1, 0, None
        U = int(B0.shape[-1])
    else:
        raise ValueError(f"B has unexpected shape {tuple(B0.shape)}")
    if U > 1 and T > 1:
        raise ValueError("actions must be provided when B has an action dimension and T > 1")
    return B0.contiguous(), int(B0.ndim == 4), U, None


def hmm_outputs(Bn: int, T: int, K: int, want, dev) -> dict:
    """Device output buffers of ``b2_hmm_smoother`` (None = not written;
    ``filtered`` always)."""
    out = {k: None for k in ("mll", "filtered", "predicted", "smoothed", "joint", "cond")}
    out["filtered"] = torch.empty((Bn, T, K), device=dev)
    if "mll" in want:
        out["mll"] = torch.empty((Bn,), device=dev)
    for k in ("predicted", "smoothed"):
        if k in want:
            out[k] = torch.empty((Bn, T, K), device=dev)
    for k in ("joint", "cond"):
        if k in want:
            out[k] = torch.empty((Bn, max(T - 1, 0), K, K), device=dev)
    return out


def hmm_smoother_packed(A_flat, A_batched: int, O, obs, distr_obs: bool, prior, B, B_batched: int, U: int, actions,
                        action_mode: str, out: dict) -> None:
    """The ``b2_hmm_smoother`` call alone on packed device buffers: ``A_flat``
    ``[Bn or 1, sum O * K]``, ``obs`` int32 ``[Bn, T, M]`` or float
    ``[Bn, T, sum O]``, ``B`` laid out for ``U`` (0 = time-varying)."""
    Bn, K = prior.shape
    T = obs.shape[1]
    ptr = lambda t: 0 if t is None else t.data_ptr()  # noqa: E731
    check(_lib.load().b2_hmm_smoother(
        _stream(prior), A_flat.data_ptr(), A_flat.numel(), int(A_batched), i64(list(O)), len(O),
        0 if distr_obs else obs.data_ptr(), obs.data_ptr() if distr_obs else 0, obs.numel(), prior.data_ptr(),
        prior.numel(), B.data_ptr(), B.numel(), int(B_batched), int(U), ptr(actions),
        0 if actions is None else actions.numel(), _MODES[action_mode], Bn, T, K, ptr(out["mll"]),
        ptr(out["filtered"]), ptr(out["predicted"]), ptr(out["smoothed"]), ptr(out["joint"]), ptr(out["cond"])))


def hmm_smoother(A, obs, prior, B0, actions=None, distr_obs=True, action_mode="index",
                 want=("mll", "filtered", "predicted", "smoothed", "cond")):
    """``b2_hmm_smoother``: ``A[m]`` ``(Bn, O_m, K)`` or ``(O_m, K)``;
    ``obs[m]`` ``(Bn, T)`` indices or ``(Bn, T, O_m)`` distributions
    (``distr_obs``); ``prior`` ``(Bn, K)``; ``B0`` as in the reference plus a
    batch axis; ``actions`` ``(Bn, T-1)``. Returns a dict of device tensors."""
    prior = _dev_f32(prior).contiguous()
    _require_cuda(prior, "prior")
    dev = prior.device
    Bn, K = prior.shape
    A = [_dev_f32(a, dev) for a in A]
    A_batched = int(A[0].ndim == 3)
    O = [int(a.shape[-2]) for a in A]
    A_flat = torch.cat([a.reshape((Bn, -1) if A_batched else (-1,)) for a in A], dim=-1).contiguous()
    if distr_obs:
        o = torch.cat([_dev_f32(x, dev).reshape(Bn, -1, O[m]) for m, x in enumerate(obs)], dim=-1).contiguous()
    else:
        o = torch.stack([torch.as_tensor(x, device=dev).reshape(Bn, -1) for x in obs], dim=-1)
        o = o.to(torch.int32).contiguous()
    T = o.shape[1]
    Bt, B_batched, U, act = _transitions(_dev_f32(B0, dev), actions, Bn, T, K)
    out = hmm_outputs(Bn, T, K, want, dev)
    hmm_smoother_packed(A_flat, A_batched, O, o, distr_obs, prior, Bt, B_batched, U, act, action_mode, out)
    return out


def run_exact_single_factor_hmm_scan(obs, A, B, prior, actions=None, distr_obs=True):
    """``pymdp/algos.py:1132-1208`` over a batch: returns
    ``(mll (Bn,), [smoothed (Bn, T, K)], [predicted (Bn, T, K)], [cond (Bn, T-1, K, K)])``."""
    if len(prior) != 1 or len(B) != 1:
        raise ValueError("run_exact_single_factor_hmm_scan expects singleton lists for prior and B")
    r = hmm_smoother(A, obs, prior[0], B[0], actions=actions, distr_obs=distr_obs)
    return r["mll"], [r["smoothed"]], [r["predicted"]], [r["cond"]]


def hmm_smoother_from_filtered_colstoch(filtered, B_mats, actions=None, return_trans_probs=False,
                                        action_mode="index"):
    """``pymdp/algos.py:1049-1130`` over a batch (``filtered`` ``(Bn, T, K)``):
    ``(smoothed, joint_next_curr, cond_probs[, trans_probs])``."""
    filtered = _dev_f32(filtered).contiguous()
    _require_cuda(filtered, "filtered")
    Bn, T, K = filtered.shape
    Bt, B_batched, U, act = _transitions(_dev_f32(B_mats, filtered.device), actions, Bn, T, K)
    dev = filtered.device
    sm = torch.empty((Bn, T, K), device=dev)
    joint = torch.empty((Bn, max(T - 1, 0), K, K), device=dev)
    cond = torch.empty_like(joint)
    check(_lib.load().b2_hmm_smoother_from_filtered(
        _stream(filtered), filtered.data_ptr(), filtered.numel(), Bt.data_ptr(), Bt.numel(), B_batched, U,
        0 if act is None else act.data_ptr(), 0 if act is None else act.numel(), _MODES[action_mode], Bn, T, K,
        sm.data_ptr(), joint.data_ptr(), cond.data_ptr()))
    if return_trans_probs:
        return sm, joint, cond, joint.transpose(-1, -2)
    return sm, joint, cond


def smoothing_exact(filtered_post, B, past_actions):
    """``pymdp/inference.py:595-634`` over a batch: ``([smoothed], [joint])``,
    a negative action being the identity transition."""
    if len(filtered_post) != 1 or len(B) != 1:
        raise ValueError("smoothing_exact currently supports only one hidden-state factor")
    sm, joint, _ = hmm_smoother_from_filtered_colstoch(filtered_post[0], B[0], actions=past_actions,
                                                       action_mode="identity")
    return [sm], [joint]


__all__ = ["hmm_smoother", "hmm_smoother_packed", "hmm_outputs", "run_exact_single_factor_hmm_scan",
           "hmm_smoother_from_filtered_colstoch", "smoothing_exact"]
