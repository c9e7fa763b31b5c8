"""``torch.autograd.Function`` wrappers over the C-ABI forward and adjoint
kernels, for model fitting.

The reference differentiates its JAX path (``pymdp/ffi/_core.py:282-310``,
``with_jax_grad``: forward through the FFI, gradient from ``jax.grad`` of the
pure-JAX function). Here both directions are native kernels:

* :class:`FpiObs`: fused-observation FPI (``b2_fpi_obs`` / ``b2_fpi_obs_bwd``),
  differentiable in the flattened A and the prior;
* :class:`NegEfe`: neg-EFE of every policy, utility + state information gain
  (``b2_neg_efe`` at FP32 / ``b2_neg_efe_bwd``), differentiable in the
  flattened qs_init, A, B and C.

Inputs are the kernels' flat layouts (``[batch, sum of per-array sizes]``);
``pymdp_b200.ffi.flatten_ragged_f32`` builds them (``torch.cat`` keeps the
autograd graph to the per-modality tensors).
"""

from __future__ import annotations

import torch

from . import _lib, ffi
from ._lib import check


class FpiObs(torch.autograd.Function):
    """``q = FPI(A_flat, prior_flat | obs)``, ``[batch, sum S]``."""

    @staticmethod
    def forward(ctx, A_flat, prior_flat, obs, A_offsets, O, S, A_dependencies, num_iter):
        A_flat, prior_flat = A_flat.contiguous(), prior_flat.contiguous()
        stride = int(A_offsets[-1]) if A_flat.ndim == 2 else 0
        q = ffi.fpi_obs_flat(A_flat, stride, A_offsets, O, obs, prior_flat, S, A_dependencies, num_iter)
        ctx.save_for_backward(A_flat, prior_flat, obs)
        ctx.meta = (stride, A_offsets, O, S, A_dependencies, num_iter)
        return q

    @staticmethod
    def backward(ctx, dq):
        A_flat, prior_flat, obs = ctx.saved_tensors
        stride, A_offsets, O, S, A_dependencies, num_iter = ctx.meta
        dq = dq.contiguous().float()
        dA = torch.empty_like(A_flat)
        dprior = torch.empty_like(prior_flat)
        dep_flat, dep_offs = ffi.flatten_dep_lists(A_dependencies)
        i64 = _lib.i64
        attrs = [i64(A_offsets), i64(O), i64(S), i64(dep_flat), i64(dep_offs)]
        check(_lib.load().b2_fpi_obs_bwd(
            ffi._stream(dq), A_flat.data_ptr(), stride, attrs[0], len(A_offsets), attrs[1], len(O), obs.data_ptr(),
            prior_flat.data_ptr(), dq.data_ptr(), dA.data_ptr(), dprior.data_ptr(), obs.shape[0], attrs[2], len(S),
            attrs[3], len(dep_flat), attrs[4], len(dep_offs), int(num_iter)))
        return dA, dprior, None, None, None, None, None, None


class NegEfe(torch.autograd.Function):
    """``G = neg_efe(qs_flat, A_flat, B_flat, C_flat)``, ``[batch, P]``
    (utility + state information gain, FP32)."""

    @staticmethod
    def forward(ctx, qs_flat, A_flat, B_flat, C_flat, policies, layout, flags):
        qs_flat, A_flat, B_flat, C_flat = (x.contiguous() for x in (qs_flat, A_flat, B_flat, C_flat))
        Bn, P = qs_flat.shape[0], policies.shape[0]
        dev = qs_flat.device
        G = torch.empty((Bn, P), device=dev)
        I_flat = torch.zeros((Bn, int(layout.I_offsets[-1])), device=dev)
        eps = torch.full((1,), 1e-3, device=dev)
        layout.call(None, policies, 0, qs_flat, A_flat, B_flat, C_flat, I_flat, None, None, eps, G, Bn, P,
                    flags & 3)
        ctx.save_for_backward(qs_flat, A_flat, B_flat, C_flat, policies)
        ctx.meta = (layout, flags & 3)
        return G

    @staticmethod
    def backward(ctx, dG):
        qs_flat, A_flat, B_flat, C_flat, policies = ctx.saved_tensors
        layout, flags = ctx.meta
        dG = dG.contiguous().float()
        Bn, P = dG.shape
        dqs, dA, dB, dC = (torch.empty_like(x) for x in (qs_flat, A_flat, B_flat, C_flat))
        c = layout._c
        check(_lib.load().b2_neg_efe_bwd(
            ffi._stream(dG), policies.data_ptr(), policies.numel(), 0, qs_flat.data_ptr(), qs_flat.numel(),
            A_flat.data_ptr(), A_flat.numel(), B_flat.data_ptr(), B_flat.numel(), C_flat.data_ptr(), C_flat.numel(),
            dG.data_ptr(), dG.numel(), dqs.data_ptr(), dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), Bn, P,
            layout.T, layout.F, layout.M, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[9], len(layout.A_dep_flat),
            c[10], c[11], len(layout.B_dep_flat), c[12], int(flags)))
        return dqs, dA, dB, dC, None, None, None
