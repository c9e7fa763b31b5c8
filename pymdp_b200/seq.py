"""Sequence inference on the GPU: batched mirrors of the reference's
``run_mmp`` / ``run_vmp`` (``pymdp/algos.py:392-430, :512-571``) over
``b2_sequence_infer``.

Same arguments as the reference with a leading batch axis on every per-agent
array: ``A[m]`` ``(batch, O_m, *S_deps)`` (or unbatched, shared), ``B[f]`` the
action-conditioned transition sequence ``(batch, T-1, S_f, *S_Bdeps)``,
``obs[m]`` ``(batch, T)`` indices (``distr_obs=False``) or ``(batch, T, O_m)``
distributions, ``prior[f]`` ``(batch, S_f)``. Returns ``qs[f]`` of shape
``(batch, T, S_f)``.
"""

from __future__ import annotations

from typing import Sequence

import numpy as np
import torch

from . import _lib
from .ffi import _require_cuda, _stream, flatten_dep_lists, i64


def _f32(x, dev):
    return torch.as_tensor(x, device=dev).to(torch.float32)


class SequencePlan:
    """The inputs of one sequence-inference call packed into the flat device
    buffers ``b2_sequence_infer`` takes (A, B, observations, prior, output and
    the dependency tables), so that ``run()`` only launches the kernel: for
    windows that are re-run on resident inputs. ``run_mmp`` / ``run_vmp``
    build one per call."""

    def __init__(self, vmp: bool, A, B, obs, prior, A_dependencies, B_dependencies, num_iter=1, tau=1.0,
                 distr_obs=True):
        dev = prior[0].device if isinstance(prior[0], torch.Tensor) else torch.device("cuda")
        prior = [_f32(p, dev) for p in prior]
        F, M = len(prior), len(A)
        if len(B) != F or len(obs) != M or len(A_dependencies) != M or len(B_dependencies) != F:
            raise ValueError("A / obs need one entry per modality, B / prior one per factor")
        Bn = int(prior[0].shape[0])
        S = [int(p.shape[-1]) for p in prior]
        A = [_f32(a, dev) for a in A]
        A_batched = A[0].ndim == len(A_dependencies[0]) + 2
        O = [int(a.shape[1 if A_batched else 0]) for a in A]
        B = [_f32(x, dev) for x in B]
        T = int(B[0].shape[1]) + 1
        for f, (x, deps) in enumerate(zip(B, B_dependencies)):
            exp = (Bn, T - 1, S[f]) + tuple(S[d] for d in deps)
            if tuple(x.shape) != exp:
                raise ValueError(f"B[{f}] shape {tuple(x.shape)} does not match {exp}")
        self.A_flat = torch.cat([a.reshape(Bn if A_batched else 1, -1) for a in A], dim=1).contiguous()
        self.B_flat = torch.cat([x.reshape(Bn, -1) for x in B], dim=1).contiguous()
        self.prior_flat = torch.cat(prior, dim=1).contiguous()
        if distr_obs:
            o = torch.cat([_f32(x, dev).reshape(Bn, T, O[m]) for m, x in enumerate(obs)], dim=2).contiguous()
            self.obs_idx, self.obs_distr = None, o
        else:
            o = torch.stack([torch.as_tensor(x, device=dev).reshape(Bn, T) for x in obs], dim=2).to(torch.int32)
            self.obs_idx, self.obs_distr = o.contiguous(), None
        self.obs = o
        self.out = torch.empty((Bn, T, sum(S)), dtype=torch.float32, device=dev)
        for t in (self.A_flat, self.B_flat, self.prior_flat, self.out, o):
            _require_cuda(t, "sequence-inference buffer")
        adf, ado = flatten_dep_lists([list(d) for d in A_dependencies])
        bdf, bdo = flatten_dep_lists([list(d) for d in B_dependencies])
        # the argument tuple of the call, built once (its ctypes arrays stay alive with the plan)
        self._args = (int(vmp), self.A_flat.data_ptr(), self.A_flat.numel(), int(A_batched), i64(O), M,
                      None if self.obs_idx is None else self.obs_idx.data_ptr(),
                      None if self.obs_distr is None else self.obs_distr.data_ptr(), o.numel(),
                      self.B_flat.data_ptr(), self.B_flat.numel(), self.prior_flat.data_ptr(), self.prior_flat.numel(),
                      self.out.data_ptr(), self.out.numel(), Bn, T, F, i64(S), i64(adf), len(adf), i64(ado),
                      i64(bdf), len(bdf), i64(bdo), int(num_iter), float(tau))
        off = np.cumsum([0] + S)
        self.qs = [self.out[:, :, off[f]:off[f + 1]] for f in range(F)]

    def run(self):
        """Launch the kernel on the packed buffers (current stream); returns
        ``qs[f]`` ``(batch, T, S_f)``, views of the plan's output buffer."""
        _lib.check(_lib.load().b2_sequence_infer(_stream(self.out), *self._args))
        return self.qs


def prepare(vmp: bool, A, B, obs, prior, A_dependencies, B_dependencies, num_iter=1, tau=1.0, distr_obs=True):
    """A ``SequencePlan`` for ``run_vmp`` (``vmp=True``) or ``run_mmp``."""
    return SequencePlan(vmp, A, B, obs, prior, A_dependencies, B_dependencies, num_iter, tau, distr_obs)


def _run(vmp: bool, A, B, obs, prior, A_dependencies, B_dependencies, num_iter=1, tau=1.0, distr_obs=True):
    return SequencePlan(vmp, A, B, obs, prior, A_dependencies, B_dependencies, num_iter, tau, distr_obs).run()


def run_mmp(A, B, obs, prior, A_dependencies: Sequence[Sequence[int]], B_dependencies: Sequence[Sequence[int]],
            num_iter: int = 1, tau: float = 1.0, distr_obs: bool = True):
    """Marginal message passing over the window (``pymdp/algos.py:392-430``)."""
    return _run(False, A, B, obs, prior, A_dependencies, B_dependencies, num_iter, tau, distr_obs)


def run_vmp(A, B, obs, prior, A_dependencies: Sequence[Sequence[int]], B_dependencies: Sequence[Sequence[int]],
            num_iter: int = 1, tau: float = 1.0, distr_obs: bool = True):
    """Variational message passing over the window (``pymdp/algos.py:512-571``)."""
    return _run(True, A, B, obs, prior, A_dependencies, B_dependencies, num_iter, tau, distr_obs)
