"""Differentiable action log-likelihood for fitting agents to behaviour.

The reference fits by scanning ``evolve_trials`` (``pymdp/likelihoods.py:7-26``)
under numpyro and differentiating it with ``jax.grad``; its FFI kernels get
their gradients from the pure-JAX path (``pymdp/ffi/_core.py:282-310``). Here
every subject is one row of a batch and each trial step runs

* ``qs = FPI(A, o_t, prior)``           — :class:`~pymdp_b200.autograd.FpiObs`
  (``b2_fpi_obs`` / ``b2_fpi_obs_bwd``);
* ``G = neg_EFE(qs, A, B, C)``           — :class:`~pymdp_b200.autograd.NegEfe`
  (``b2_neg_efe`` / ``b2_neg_efe_bwd``);
* ``q_pi = softmax(gamma G + log E)``    (``pymdp/control.py:349``);
* ``probs = multiaction_probabilities``  (``pymdp/agent.py:908-937``,
  ``sampling_mode="full"``);
* ``prior = B[..., a_t] . qs``           (``pymdp/agent.py:825-851``).

Parameters are the softmax logits of A (over observations) and B (over next
states), C (log preferences, the same at every policy step) and ``log gamma``,
each with a leading subject axis. ``form="log"`` scores ``log probs[a_t]``;
``form="probs_as_logits"`` scores ``log_softmax(probs)[a_t]``, which is what
``aif_likelihood`` (``pymdp/likelihoods.py:28-45``) computes when it passes the
probabilities to ``Categorical(logits=...)``.
"""

from __future__ import annotations

import math
from typing import Sequence

import numpy as np
import torch

from . import ffi
from .autograd import FpiObs, NegEfe
from .control import construct_policies


class FitModel:
    """Structure of the fitted generative model, shared by every subject.

    Transitions are factor-local (``B_f`` is ``(S_f, S_f, U_f)``), which is
    what ``update_empirical_prior`` assumes (``pymdp/control.py:377-378``).
    """

    def __init__(self, num_states: Sequence[int], num_obs: Sequence[int], num_controls: Sequence[int],
                 policy_len: int = 1, A_dependencies: Sequence[Sequence[int]] | None = None, num_iter: int = 16,
                 device="cuda"):
        self.S = [int(s) for s in num_states]
        self.O = [int(o) for o in num_obs]
        self.U = [int(u) for u in num_controls]
        self.F, self.M = len(self.S), len(self.O)
        self.policy_len = int(policy_len)
        self.num_iter = int(num_iter)
        self.device = torch.device(device)
        self.A_dependencies = ([list(range(self.F))] * self.M if A_dependencies is None
                               else [list(map(int, d)) for d in A_dependencies])
        self.B_dependencies = [[f] for f in range(self.F)]
        self.A_shapes = [(o,) + tuple(self.S[d] for d in deps) for o, deps in zip(self.O, self.A_dependencies)]
        self.B_shapes = [(s, s, u) for s, u in zip(self.S, self.U)]
        pol = construct_policies(self.S, self.U, self.policy_len)
        self.P = pol.shape[0]
        self.policies = torch.as_tensor(pol, device=self.device)
        self.layout = ffi.EfeLayout(self.S, self.O, self.U, self.policy_len, self.A_dependencies,
                                    self.B_dependencies)
        self.A_offsets = self.layout.A_offsets
        # multi-action of each policy's first step, row-major over num_controls
        k = np.zeros(self.P, dtype=np.int64)
        for f, u in enumerate(self.U):
            k = k * u + pol[:, 0, f]
        self.n_multi = int(np.prod(self.U))
        onehot = np.zeros((self.P, self.n_multi), dtype=np.float32)
        onehot[np.arange(self.P), k] = 1.0
        self.policy_to_multi = torch.as_tensor(onehot, device=self.device)
        self.log_E = torch.full((self.P,), -math.log(self.P), device=self.device)
        self.qs_offsets = np.cumsum([0] + self.S)
        self.multi_stride = torch.as_tensor([int(np.prod(self.U[f + 1:])) for f in range(self.F)],
                                            device=self.device)

    # ------------------------------------------------------------------ params
    def init_params(self, n_subjects: int, generator: torch.Generator | None = None, log_gamma_mean=math.log(8.0),
                    log_gamma_std=0.3):
        """Logits ~ N(0, 1), C ~ N(0, 1), log gamma ~ N(mean, std)."""
        kw = dict(device=self.device, generator=generator)
        A = [torch.randn((n_subjects,) + s, **kw) for s in self.A_shapes]
        B = [torch.randn((n_subjects,) + s, **kw) for s in self.B_shapes]
        C = [torch.randn((n_subjects, o), **kw) for o in self.O]
        lg = log_gamma_mean + log_gamma_std * torch.randn((n_subjects,), **kw)
        return A, B, C, lg

    def _flat_model(self, A_logits, B_logits, C):
        n = A_logits[0].shape[0]
        A = [torch.softmax(a, dim=1) for a in A_logits]
        B = [torch.softmax(b, dim=1) for b in B_logits]
        A_flat = torch.cat([a.reshape(n, -1) for a in A], dim=1)
        B_flat = torch.cat([b.reshape(n, -1) for b in B], dim=1)
        C_flat = torch.cat([c[:, None, :].expand(n, self.policy_len, c.shape[1]).reshape(n, -1) for c in C], dim=1)
        return A_flat, B, B_flat, C_flat

    def _prior_next(self, B, qs, a_t):
        out = []
        for f in range(self.F):
            q = qs[:, self.qs_offsets[f]:self.qs_offsets[f + 1]]
            Bf = B[f].permute(0, 3, 1, 2)  # (n, U, S, S)
            Bsel = Bf[torch.arange(Bf.shape[0], device=Bf.device), a_t[:, f]]
            out.append(torch.bmm(Bsel, q.unsqueeze(-1)).squeeze(-1))
        return torch.cat(out, dim=1)

    def _step_probs(self, A_flat, B_flat, C_flat, gamma, prior, o_t):
        qs = FpiObs.apply(A_flat, prior, o_t, self.A_offsets, self.O, self.S, self.A_dependencies, self.num_iter)
        G = NegEfe.apply(qs, A_flat, B_flat, C_flat, self.policies, self.layout, 3)
        q_pi = torch.softmax(gamma[:, None] * G + self.log_E, dim=-1)
        return qs, q_pi @ self.policy_to_multi

    # -------------------------------------------------------------- likelihood
    def log_likelihood(self, A_logits, B_logits, C, log_gamma, obs, actions, form: str = "log",
                       per_subject: bool = False):
        """Summed action log-likelihood.

        ``obs``: ``(T, n, M)`` int32, ``actions``: ``(T, n, F)`` int64 (time
        major, on the model's device). Returns a scalar (or ``(n,)`` with
        ``per_subject``) that ``backward()`` differentiates w.r.t. every
        parameter through the native adjoints.
        """
        if form not in ("log", "probs_as_logits"):
            raise ValueError("form must be 'log' or 'probs_as_logits'")
        A_flat, B, B_flat, C_flat = self._flat_model(A_logits, B_logits, C)
        n = A_flat.shape[0]
        gamma = torch.exp(log_gamma)
        prior = torch.cat([torch.full((n, s), 1.0 / s, device=A_flat.device) for s in self.S], dim=1)
        ll = torch.zeros(n, device=A_flat.device)
        for t in range(obs.shape[0]):
            qs, probs = self._step_probs(A_flat, B_flat, C_flat, gamma, prior, obs[t])
            k = (actions[t] * self.multi_stride).sum(-1, keepdim=True)
            lp = torch.log(probs) if form == "log" else torch.log_softmax(probs, dim=-1)
            ll = ll + lp.gather(1, k).squeeze(1)
            prior = self._prior_next(B, qs, actions[t])
        return ll if per_subject else ll.sum()

    # -------------------------------------------------------------- simulation
    @torch.no_grad()
    def simulate(self, A_logits, B_logits, C, log_gamma, T: int, generator: torch.Generator | None = None):
        """Roll each subject's agent out in an environment that is its own
        generative model: hidden states from D (uniform) and B, observations
        from A, actions sampled from the agent's multi-action probabilities.
        Returns ``(obs (T, n, M) int32, actions (T, n, F) int64)``."""
        A_flat, B, B_flat, C_flat = self._flat_model(A_logits, B_logits, C)
        A = [torch.softmax(a, dim=1) for a in A_logits]
        n = A_flat.shape[0]
        dev = A_flat.device
        ar = torch.arange(n, device=dev)
        gamma = torch.exp(log_gamma)
        prior = torch.cat([torch.full((n, s), 1.0 / s, device=dev) for s in self.S], dim=1)
        s = torch.stack([torch.multinomial(torch.full((n, sf), 1.0 / sf, device=dev), 1, generator=generator)[:, 0]
                         for sf in self.S], dim=1)
        obs = torch.empty((T, n, self.M), dtype=torch.int32, device=dev)
        acts = torch.empty((T, n, self.F), dtype=torch.int64, device=dev)
        div = [int(np.prod(self.U[f + 1:])) for f in range(self.F)]
        for t in range(T):
            for m, deps in enumerate(self.A_dependencies):
                col = A[m][(ar, slice(None)) + tuple(s[:, d] for d in deps)]  # (n, O_m)
                obs[t, :, m] = torch.multinomial(col, 1, generator=generator)[:, 0].to(torch.int32)
            qs, probs = self._step_probs(A_flat, B_flat, C_flat, gamma, prior, obs[t])
            k = torch.multinomial(probs.clamp_min(0), 1, generator=generator)[:, 0]
            for f in range(self.F):
                acts[t, :, f] = (k // div[f]) % self.U[f]
            prior = self._prior_next(B, qs, acts[t])
            s = torch.stack([torch.multinomial(B[f][ar, :, s[:, f], acts[t, :, f]], 1, generator=generator)[:, 0]
                             for f in range(self.F)], dim=1)
        return obs, acts


class GraphedLogLikelihood:
    """One forward + backward of :meth:`FitModel.log_likelihood` over fixed
    trials, captured in a CUDA graph.

    ``params`` are leaf tensors (A logits, B logits, C, log gamma, in that
    order, as lists flattened into one list) that the caller updates IN
    PLACE between calls; each call replays the graph and returns the static
    likelihood tensor, with the gradients in ``p.grad`` (overwritten, not
    accumulated). Every kernel of the step, the native FPI / neg-EFE forward
    and adjoint launches included, is replayed without host work. No earlier
    autograd graph over ``params`` may still be alive at construction (drop
    any eager loss first): its gradient-accumulation nodes belong to another
    stream and break the capture.
    """

    def __init__(self, model: FitModel, params: Sequence[torch.Tensor], obs, actions, form: str = "log",
                 warmup: int = 3):
        self.model, self.params = model, list(params)
        nA, nB, nC = model.M, model.F, model.M
        if len(self.params) != nA + nB + nC + 1:
            raise ValueError("params must be A logits + B logits + C + [log_gamma]")
        self.obs, self.actions = obs.contiguous(), actions.contiguous()
        split = (self.params[:nA], self.params[nA:nA + nB], self.params[nA + nB:nA + nB + nC], self.params[-1])

        def step():
            ll = model.log_likelihood(*split, self.obs, self.actions, form=form)
            ll.backward()
            return ll

        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(warmup):
                for p in self.params:
                    p.grad = None
                step()
        torch.cuda.current_stream().wait_stream(side)
        for p in self.params:
            p.grad = None
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.ll = step()

    def __call__(self) -> torch.Tensor:
        self.graph.replay()
        return self.ll
