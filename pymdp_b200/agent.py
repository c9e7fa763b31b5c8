"""``Agent`` — the reference's ``pymdp.agent.Agent`` surface for the FPI + EFE path.

Keeps the signatures and return shapes of ``Agent.infer_states``
(``pymdp/agent.py:675-823``), ``Agent.infer_policies`` (``:853-906``),
``Agent.sample_action`` (``:939-967``) and ``Agent.infer_parameters``
(``:416-620``, Dirichlet learning of A and B) for ``inference_algo="fpi"``,
either ``sampling_mode`` and either action selection, with the
batch-broadcasting rules of ``pymdp/agent.py:228-330`` (unbatched A/B/C/D/E
are broadcast to ``batch_size``; defaults C = uniform 1/O, D = uniform,
E = uniform).

Model tensors are flattened ONCE into device buffers at construction (the
reference re-flattens A/B/C on every call, ``pymdp/ffi/_efe.py:596-613``), so
each call is a handful of kernel launches on the current stream and nothing
else.
"""

from __future__ import annotations

import ctypes

from typing import Sequence

import numpy as np
import torch

from . import ffi
from .control import construct_policies, generate_I_matrix


def _views(flat: torch.Tensor, offsets, shapes) -> list[torch.Tensor]:
    """Per-array views ``[batch, *shape]`` of a flattened ``[batch, total]`` buffer."""
    return [flat[:, int(offsets[i]):int(offsets[i + 1])].unflatten(1, tuple(sh)) for i, sh in enumerate(shapes)]


def _t(x, dev) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=torch.float32)
    return torch.as_tensor(np.asarray(x, dtype=np.float32), device=dev)


class Agent:
    """Batched active-inference agent whose hot paths run on sm_100a kernels."""

    def __init__(self, A: Sequence, B: Sequence, C: Sequence | None = None, D: Sequence | None = None,
                 E=None, A_dependencies: Sequence[Sequence[int]] | None = None,
                 B_dependencies: Sequence[Sequence[int]] | None = None, num_controls=None, policy_len: int = 1,
                 policies=None, control_fac_idx=None, gamma: float = 1.0, alpha: float = 1.0,
                 use_utility: bool = True, use_states_info_gain: bool = True, use_param_info_gain: bool = False,
                 use_inductive: bool = False, action_selection: str = "deterministic",
                 sampling_mode: str = "full", inference_algo: str = "fpi", num_iter: int = 16,
                 batch_size: int = 1, precision: str = "fp32", device="cuda", pA: Sequence | None = None,
                 pB: Sequence | None = None, H: Sequence | None = None, I: Sequence | None = None,
                 inductive_depth: int = 1, inductive_threshold: float = 0.1, inductive_epsilon=1e-3,
                 learn_A: bool = False, learn_B: bool = False, efe_algorithm: str = "factored"):
        if inference_algo.lower() != "fpi":
            raise NotImplementedError("only inference_algo='fpi' is on the accelerated path")
        if use_param_info_gain and pA is None and pB is None:
            raise ValueError("use_param_info_gain=True requires at least one of pA or pB.")
        if learn_A and pA is None:
            raise ValueError("pA is required for A learning")
        if learn_B and pB is None:
            raise ValueError("pB is required for B learning")
        if use_inductive and inductive_depth < 1:
            raise ValueError("`inductive_depth` must be >= 1")
        if action_selection not in ("deterministic", "stochastic"):
            raise ValueError("action_selection must be 'deterministic' or 'stochastic'")
        if sampling_mode not in ("full", "marginal"):
            raise ValueError("sampling_mode must be 'full' or 'marginal'")
        if efe_algorithm not in ("factored", "dense"):
            raise ValueError("efe_algorithm must be 'factored' or 'dense'")
        dev = torch.device(device)
        self.device = dev
        self.batch_size = int(batch_size)
        self.num_iter = int(num_iter)
        self.precision = precision
        self.use_utility, self.use_states_info_gain = use_utility, use_states_info_gain
        self.action_selection, self.sampling_mode = action_selection, sampling_mode
        M, F = len(A), len(B)
        self.num_modalities, self.num_factors = M, F
        self.A_dependencies = [list(d) for d in (A_dependencies or [list(range(F)) for _ in range(M)])]
        self.B_dependencies = [list(d) for d in (B_dependencies or [[f] for f in range(F)])]
        A = [_t(a, dev) for a in A]
        B = [_t(b, dev) for b in B]
        # num_states from B (pymdp/agent.py:399-414: the self-dependency axis)
        S = []
        for f, deps in enumerate(self.B_dependencies):
            if f not in deps:
                raise ValueError(f"num_states cannot be inferred from B, B_dependencies if the dynamics of "
                                 f"hidden state {f} is not conditioned on itself")
            S.append(int(B[f].shape[-(len(deps) + 1 - deps.index(f))]))
        self.num_states = S
        nbat = self.batch_size

        def batched(x, core_ndim, name):
            if x.ndim == core_ndim + 1:
                if x.shape[0] == 1 and nbat > 1:
                    return x.expand((nbat,) + tuple(x.shape[1:]))
                if x.shape[0] != nbat:
                    raise ValueError(f"Batch size {nbat} does not match the first dimension of {name} with shape "
                                     f"{tuple(x.shape)}")
                return x
            if x.ndim == core_ndim:
                return x.unsqueeze(0).expand((nbat,) + tuple(x.shape))
            raise ValueError(f"{name} has unexpected shape {tuple(x.shape)}")

        # C follows A's batching (pymdp/agent.py:278-294): broadcast when A[m] was unbatched
        A_was_batched = [a.ndim == len(self.A_dependencies[m]) + 2 for m, a in enumerate(A)]
        A = [batched(a, len(self.A_dependencies[m]) + 1, f"A[{m}]") for m, a in enumerate(A)]
        B = [batched(b, len(self.B_dependencies[f]) + 2, f"B[{f}]") for f, b in enumerate(B)]
        self.num_obs = [int(a.shape[1]) for a in A]
        self.num_controls = [int(b.shape[-1]) for b in B]
        if control_fac_idx is None:
            control_fac_idx = [f for f in range(F) if self.num_controls[f] > 1]
        self.control_fac_idx = list(control_fac_idx)
        self.policy_len = int(policy_len)
        pol = construct_policies(S, self.num_controls, self.policy_len, self.control_fac_idx) \
            if policies is None else np.asarray(policies, dtype=np.int32)
        self.policies = torch.as_tensor(pol, device=dev, dtype=torch.int32).contiguous()
        P = int(pol.shape[0])
        if C is None:
            C = [torch.full((nbat, o), 1.0 / o, device=dev) for o in self.num_obs]
        else:
            C = [_t(c, dev) for c in C]
            C = [c if A_was_batched[m] and c.shape[0] == nbat else
                 (c.expand((nbat,) + tuple(c.shape[1:])) if A_was_batched[m] else
                  c.unsqueeze(0).expand((nbat,) + tuple(c.shape)))
                 for m, c in enumerate(C)]
        if D is None:
            D = [torch.full((nbat, s), 1.0 / s, device=dev) for s in S]
        else:
            D = [batched(_t(d, dev), 1, f"D[{f}]") for f, d in enumerate(D)]
        if E is None:
            E = torch.full((nbat, P), 1.0 / P, device=dev)
        else:
            E = batched(_t(E, dev), 1, "E")
        self.D = [d.contiguous() for d in D]
        self.E = E.contiguous()
        self.gamma = _t(np.broadcast_to(np.asarray(gamma, np.float32), (nbat,)).copy(), dev)
        self.alpha = _t(np.broadcast_to(np.asarray(alpha, np.float32), (nbat,)).copy(), dev)
        # one-time flattening into the kernels' layouts
        self._A_flat, self._A_offsets = ffi.flatten_ragged_f32(A, 1, dev)
        self._B_flat, _ = ffi.flatten_ragged_f32(B, 1, dev)
        C_t = []
        for m, c in enumerate(C):
            if c.ndim == 2:  # (batch, O)
                c = c.unsqueeze(1).expand(nbat, self.policy_len, self.num_obs[m])
            C_t.append(c)
        self._C_flat, _ = ffi.flatten_ragged_f32(C_t, 1, dev)
        self._qs_offsets = np.cumsum([0] + S)
        # inductive matrices (pymdp/agent.py:368-380): from H via generate_I_matrix, or given
        if use_inductive and H is not None:
            H_b = [np.broadcast_to(np.asarray(_t(h, "cpu")), (nbat, S[f])) for f, h in enumerate(H)]
            per_agent = [generate_I_matrix([H_b[f][b_] for f in range(F)], [B[f][b_].cpu().numpy() for f in range(F)],
                                           float(inductive_threshold), int(inductive_depth)) for b_ in range(nbat)]
            I = [torch.as_tensor(np.stack([per_agent[b_][f] for b_ in range(nbat)]), device=dev) for f in range(F)]
        elif use_inductive and I is not None:
            I = [batched(_t(i, dev), 2, f"I[{f}]") for f, i in enumerate(I)]
        else:
            I = [torch.zeros((nbat, 1, s), device=dev) for s in S]
        self.I = I
        self._layout = ffi.EfeLayout(S, self.num_obs, self.num_controls, self.policy_len, self.A_dependencies,
                                     self.B_dependencies, [int(i.shape[1]) for i in I])
        self._I_flat, _ = ffi.flatten_ragged_f32(I, 1, dev)
        self._eps = _t(np.broadcast_to(np.asarray(inductive_epsilon, np.float32), (nbat,)).copy(), dev)
        # Dirichlet parameters (pymdp/agent.py:201-250); a None entry of pA is a
        # modality that neither informs the parameter information gain nor learns
        self._pA_mask = 0 if pA is None else sum(1 << m for m, x in enumerate(pA) if x is not None)
        if use_param_info_gain and pA is not None and self._pA_mask != (1 << M) - 1:
            raise NotImplementedError("use_param_info_gain with a None entry in pA")
        pA_b = None if pA is None else [
            A[m] * 0 if x is None else batched(_t(x, dev), len(self.A_dependencies[m]) + 1, f"pA[{m}]")
            for m, x in enumerate(pA)]
        pB_b = None if pB is None else [batched(_t(x, dev), len(self.B_dependencies[f]) + 2, f"pB[{f}]")
                                        for f, x in enumerate(pB)]
        self._pA_flat = ffi.flatten_ragged_f32(pA_b, 1, dev)[0] if pA_b is not None else None
        self._pB_flat = ffi.flatten_ragged_f32(pB_b, 1, dev)[0] if pB_b is not None else None
        self.learn_A, self.learn_B = bool(learn_A), bool(learn_B)
        self._H = H if (use_inductive and H is not None) else None
        self.inductive_depth, self.inductive_threshold = int(inductive_depth), float(inductive_threshold)
        # policies built here are construct_policies' full product set: let the
        # tensor-core paths share the evaluation of common policy prefixes
        # and, with factor-local transitions, the factored contraction
        # (efe_algorithm="factored"; the flag is ignored where it cannot apply)
        self.efe_algorithm = efe_algorithm
        self._flags = ffi.efe_flags(use_utility, use_states_info_gain, use_param_info_gain, use_inductive,
                                    precision=precision, policy_tree=policies is None,
                                    factored=efe_algorithm == "factored")
        self.use_param_info_gain, self.use_inductive = use_param_info_gain, use_inductive
        # A, B (and pA, pB) are views of the flattened buffers the kernels read,
        # so learning updates them in place
        self._B_offsets = np.cumsum([0] + [int(np.prod(b.shape[1:])) for b in B])
        self.A = _views(self._A_flat, self._A_offsets, [a.shape[1:] for a in A])
        self.B = _views(self._B_flat, self._B_offsets, [b.shape[1:] for b in B])
        self.pA = None if pA is None else [
            None if x is None else v
            for x, v in zip(pA, _views(self._pA_flat, self._A_offsets, [a.shape[1:] for a in A]))]
        self.pB = None if pB is None else _views(self._pB_flat, self._B_offsets, [b.shape[1:] for b in B])
        self.C = C

    def _pack_cache(self, P: int):
        """The tensor-core operand images of this agent's (immutable) A and C,
        packed on the first call and reused (``b2_neg_efe_cached``); None
        when the call takes the SIMT path."""
        if not hasattr(self, "_pack"):
            n = self._layout.pack_bytes(self.batch_size, P, self._flags)
            self._pack = None if n == 0 else (torch.empty(n, dtype=torch.uint8, device=self.device),
                                              ctypes.c_int32(0))
        return self._pack

    # ------------------------------------------------------------------ API
    def infer_states(self, observations, empirical_prior: Sequence[torch.Tensor]):
        """``pymdp/agent.py:675-823`` (fpi): returns ``qs[f]`` of shape ``(batch, 1, S_f)``.

        ``observations``: list of M index arrays of shape ``(batch,)`` (or a
        ``(batch, M)`` array) — discrete observations, one-hot in the reference.
        """
        if not isinstance(empirical_prior, (list, tuple)):
            raise ValueError("`empirical_prior` must be a list/tuple with one entry per hidden-state factor.")
        if len(empirical_prior) != self.num_factors:
            raise ValueError(f"`empirical_prior` has {len(empirical_prior)} factor(s), expected {self.num_factors}")
        dev = self.device
        if isinstance(observations, (list, tuple)):
            obs = torch.stack([torch.as_tensor(o, device=dev).reshape(-1) for o in observations], dim=-1)
        else:
            obs = torch.as_tensor(observations, device=dev)
        obs = obs.to(torch.int32).reshape(self.batch_size, self.num_modalities).contiguous()
        prior_flat, _ = ffi.flatten_ragged_f32(
            [torch.broadcast_to(_t(p, dev), (self.batch_size, self.num_states[f]))
             for f, p in enumerate(empirical_prior)], 1, dev)
        q = self._fpi_flat(obs, prior_flat)
        o = self._qs_offsets
        return [q[:, o[f]:o[f + 1]].unsqueeze(1) for f in range(self.num_factors)]

    def _fpi_flat(self, obs: torch.Tensor, prior_flat: torch.Tensor, out=None) -> torch.Tensor:
        """Fused FPI on flat ``(batch, M)`` int32 observations and a flat
        ``(batch, sum S)`` prior: the flat posterior ``(batch, sum S)``."""
        return ffi.fpi_obs_flat(self._A_flat, int(self._A_offsets[-1]), self._A_offsets, self.num_obs, obs,
                                prior_flat, self.num_states, self.A_dependencies, self.num_iter, out=out)

    def _policies_flat(self, qs_flat: torch.Tensor):
        """neg-EFE of every policy and q_pi from the flat ``(batch, sum S)`` posterior."""
        P = self.policies.shape[0]
        G = torch.empty((self.batch_size, P), device=self.device)
        pig = self.use_param_info_gain
        self._layout.call(None, self.policies, 0, qs_flat, self._A_flat, self._B_flat, self._C_flat,
                          self._I_flat, self._pA_flat if pig else None, self._pB_flat if pig else None, self._eps, G,
                          self.batch_size, P, self._flags, cache=self._pack_cache(P))
        return ffi.policy_posterior(G, self.E, self.gamma), G

    def infer_policies(self, qs: Sequence[torch.Tensor]):
        """``pymdp/agent.py:853-906``: returns ``(q_pi, neg_efe)``, each ``(batch, P)``."""
        latest = [q[:, -1] if q.ndim == 3 else q for q in qs]
        qs_flat, _ = ffi.flatten_ragged_f32(latest, 1, self.device)
        return self._policies_flat(qs_flat)

    def sample_action(self, q_pi: torch.Tensor, rng_key=None) -> torch.Tensor:
        """``pymdp/agent.py:939-967``: ``(batch, F)`` int32 actions by this
        agent's ``sampling_mode`` and ``action_selection``. For stochastic
        selection ``rng_key`` is an integer seed (a counter-based generator
        stands in for JAX's key)."""
        if self.sampling_mode == "full" and self.action_selection == "deterministic":
            return ffi.select_action(q_pi, self.policies)
        return ffi.sample_action(q_pi, self.policies, self.num_controls, self.sampling_mode, self.action_selection,
                                 self.alpha, rng_key)

    def capture_step(self, warmup: int = 2, split: bool = False) -> "GraphedAgentStep":
        """The agent step ``infer_states`` -> ``infer_policies`` ->
        ``sample_action`` as one CUDA graph over static buffers
        (``GraphedAgentStep``): a replay is one host call for the whole step
        (two with ``split``: the belief update, then policies and action)."""
        return GraphedAgentStep(self, warmup, split)

    def capture_pipeline(self, warmup: int = 2) -> "PipelinedAgentStep":
        """The graphed agent step over two buffer sets that successive steps
        alternate between (``PipelinedAgentStep``): a step's host inputs are
        copied in, and its action copied out, on copy streams while the GPU
        computes the neighbouring steps."""
        return PipelinedAgentStep(self, warmup)

    def update_empirical_prior(self, action, qs: Sequence[torch.Tensor]):
        """``pymdp/agent.py:825-851`` for ``inference_algo="fpi"``: the prior of
        the next ``infer_states``, ``compute_expected_state`` of the latest
        posterior under the sampled ``action`` (``(batch, F)`` int), per agent
        on the device (``b2_expected_state``). Returns ``pred[f]`` of shape
        ``(batch, S_f)``."""
        latest = [q[:, -1] if q.ndim == 3 else q for q in qs]
        qs_flat, _ = ffi.flatten_ragged_f32(latest, 1, self.device)
        act = torch.as_tensor(action, device=self.device).to(torch.int32).reshape(self.batch_size,
                                                                                   self.num_factors)
        pred = ffi.expected_state(qs_flat, self._B_flat, act, self._layout)
        o = self._qs_offsets
        return [pred[:, o[f]:o[f + 1]] for f in range(self.num_factors)]

    @property
    def unique_multiactions(self) -> torch.Tensor:
        """``pymdp/agent.py:396-399``: the distinct first-step joint actions of the
        policies (sorted), padded with -1 rows to ``prod(num_controls)``."""
        if not hasattr(self, "_unique"):
            self._unique = torch.as_tensor(ffi.unique_multiactions(self.policies.cpu().numpy(), self.num_controls),
                                           device=self.device)
        return self._unique

    def multiaction_probabilities(self, q_pi: torch.Tensor) -> torch.Tensor:
        """``pymdp/agent.py:908-937``: probabilities of the unique multi-actions,
        ``(batch, prod(num_controls))``: q_pi summed over the policies that
        start with each one ("full"), or the outer product of the per-factor
        action marginals ("marginal"), on the device."""
        return ffi.multiaction_probabilities(q_pi, self.policies, self.unique_multiactions, self.num_controls,
                                             self.sampling_mode)

    def infer_parameters(self, beliefs_A, observations, actions, beliefs_B=None, lr_pA=1.0, lr_pB=1.0,
                         joint_beliefs=None):
        """``pymdp/agent.py:416-620`` for ``inference_algo="fpi"``: Dirichlet
        updates of pA -> A (``learn_A``) and pB -> B (``learn_B``), in place on
        the device buffers (``b2_update_obs_likelihood_dirichlet``,
        ``b2_update_state_transition_dirichlet``); returns ``self``.

        ``beliefs_A[f]``: ``(batch, T, S_f)`` (or ``(batch, S_f)``, T = 1);
        ``observations``: per modality ``(batch,)`` / ``(batch, T)`` indices, or
        float ``(batch, T, O_m)`` distributions (categorical observations);
        ``actions``: ``(batch, F)`` or ``(batch, T', F)``, sliced to T-1 steps
        of the B belief sequence (``beliefs_B`` if given, else ``beliefs_A``).
        B learns only when some agent of the batch has a transition whose
        actions are all >= 0 (``agent.py:480-500``); with ``use_inductive``
        and H, I is then regenerated from the new B (``agent.py:606-615``).
        ``joint_beliefs[f]``: ``(batch, T-1, S_f, *S[B_dependencies[f]])``
        pairwise posteriors (e.g. from ``hmm.smoothing_exact``): B then learns
        from them, as the smoothing algorithms' branch does
        (``agent.py:530-567``), instead of from outer products of
        ``beliefs_B``."""
        dev, nbat = self.device, self.batch_size

        def seq(beliefs):
            qs = [_t(q, dev) for q in beliefs]
            qs = [q.reshape(nbat, -1, self.num_states[f]) for f, q in enumerate(qs)]
            return torch.cat(qs, dim=-1).contiguous()

        def rate(lr):
            return _t(np.broadcast_to(np.asarray(lr, np.float32), (nbat,)).copy(), dev) \
                if not isinstance(lr, torch.Tensor) else lr.to(dev, torch.float32).expand(nbat).contiguous()

        if self.learn_A:
            qa = seq(beliefs_A)
            T = qa.shape[1]
            obs = [torch.as_tensor(o, device=dev) for o in (observations if isinstance(observations, (list, tuple))
                                                             else list(torch.as_tensor(observations).unbind(-1)))]
            categorical = obs[0].is_floating_point()
            if categorical:
                o = torch.cat([x.to(torch.float32).reshape(nbat, T, self.num_obs[m]) for m, x in enumerate(obs)], -1)
            else:
                o = torch.stack([x.reshape(nbat, T) for x in obs], dim=-1).to(torch.int32)
            self._layout.learn_A(self._pA_flat, self._A_flat, o.contiguous(), qa, rate(lr_pA), nbat, T,
                                 modality_mask=self._pA_mask, categorical=categorical)
        if self.learn_B and actions is not None and joint_beliefs is not None:
            joint = torch.cat([_t(j, dev).reshape(nbat, -1) for j in joint_beliefs], dim=1).contiguous()
            T = int(_t(joint_beliefs[0], dev).shape[1]) + 1
            act = torch.as_tensor(actions, device=dev).to(torch.int32)
            if act.ndim == 2:
                act = act.unsqueeze(1)
            act = act[:, :T - 1].contiguous()
            if T > 1 and act.shape[1] == T - 1:
                if not hasattr(self, "_learn_work"):
                    self._learn_work = torch.zeros(1, dtype=torch.int32, device=dev)
                self._layout.learn_B_joint(self._pB_flat, self._B_flat, joint, act, rate(lr_pB), self._learn_work,
                                           nbat, T)
                if self._H is not None and bool((act >= 0).all(dim=-1).any()):
                    self._regenerate_I()
        elif self.learn_B and actions is not None:
            qb = seq(beliefs_A if beliefs_B is None else beliefs_B)
            T = qb.shape[1]
            act = torch.as_tensor(actions, device=dev).to(torch.int32)
            if act.ndim == 2:
                act = act.unsqueeze(1)
            act = act[:, :max(T - 1, 0)].contiguous()
            if T > 1 and act.shape[1] == T - 1:
                if not hasattr(self, "_learn_work"):
                    self._learn_work = torch.zeros(1, dtype=torch.int32, device=dev)
                self._layout.learn_B(self._pB_flat, self._B_flat, qb, act, rate(lr_pB), self._learn_work, nbat, T)
                # B is unchanged when no agent had a valid transition: keep I
                if self._H is not None and bool((act >= 0).all(dim=-1).any()):
                    self._regenerate_I()
        if getattr(self, "_pack", None) is not None:  # the tensor-core operand images hold the old A
            self._pack[1].value = 0
        return self

    def _regenerate_I(self):
        """``control.generate_I_matrix`` on the learned B (``agent.py:606-615``);
        a host computation, as in the constructor."""
        F, nbat = self.num_factors, self.batch_size
        H_b = [np.broadcast_to(np.asarray(_t(h, "cpu")), (nbat, self.num_states[f])) for f, h in enumerate(self._H)]
        B_host = [b.cpu().numpy() for b in self.B]
        per = [generate_I_matrix([H_b[f][b_] for f in range(F)], [B_host[f][b_] for f in range(F)],
                                 self.inductive_threshold, self.inductive_depth) for b_ in range(nbat)]
        I = [torch.as_tensor(np.stack([per[b_][f] for b_ in range(nbat)]), device=self.device, dtype=torch.float32)
             for f in range(F)]
        if [int(i.shape[1]) for i in I] != [int(d) for d in self._layout.I_depths]:
            raise NotImplementedError("the learned B changed the inductive depth of I")
        self.I = I
        self._I_flat, _ = ffi.flatten_ragged_f32(I, 1, self.device)


class GraphedAgentStep:
    """One agent step of ``agent`` — fused FPI, neg-EFE of every policy, q_pi
    and the action — captured once in a CUDA graph and replayed.

    The graph reads two static input buffers, ``obs`` (``(batch, M)`` int32)
    and ``prior`` (``(batch, sum S)`` float32, factor-major like the flat
    posterior), and writes four static outputs, ``qs`` (per-factor views of
    ``(batch, 1, S_f)``), ``q_pi``, ``G`` (``(batch, P)``) and ``action``
    (``(batch, F)`` int32). ``step`` copies new inputs into the buffers (on
    the current stream), replays the graph and returns the outputs, which
    the next replay overwrites. The model buffers (A, B, C, ...) are read in
    place, so in-place learning between replays is seen by the next one.
    Deterministic action selection only: a stochastic draw would replay the
    key it was captured with. ``split=True`` captures two graphs, the belief
    update and then policies + action (``graphs``), so that a caller can
    time or interleave them; ``step`` replays both.
    """

    def __init__(self, agent: Agent, warmup: int = 2, split: bool = False):
        if agent.action_selection != "deterministic":
            raise ValueError("capture_step needs action_selection='deterministic' (a replay reuses its captured key)")
        dev = agent.device
        self.agent = agent
        B, S = agent.batch_size, agent.num_states
        self.obs = torch.zeros((B, agent.num_modalities), dtype=torch.int32, device=dev)
        self.prior = torch.cat([torch.full((B, s), 1.0 / s, device=dev) for s in S], dim=1).contiguous()
        self._post = torch.empty_like(self.prior)
        self.stream = torch.cuda.Stream(dev)

        def states():
            agent._fpi_flat(self.obs, self.prior, out=self._post)

        def policies():
            q_pi, G = agent._policies_flat(self._post)
            return q_pi, G, agent.sample_action(q_pi)

        self.stream.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(self.stream):
            for _ in range(max(int(warmup), 1)):  # first calls build the per-model caches outside the capture
                states()
                policies()
        self.stream.synchronize()
        if split:
            g_states, g_policies = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
            with torch.cuda.graph(g_states, stream=self.stream):
                states()
            with torch.cuda.graph(g_policies, stream=self.stream):
                self.q_pi, self.G, self.action = policies()
            self.graphs = (g_states, g_policies)
        else:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=self.stream):
                states()
                self.q_pi, self.G, self.action = policies()
            self.graphs = (g,)
        o = agent._qs_offsets
        self.qs = [self._post[:, o[f]:o[f + 1]].unsqueeze(1) for f in range(agent.num_factors)]

    def step(self, observations=None, empirical_prior=None):
        """Replay the step; returns ``(qs, q_pi, G, action)`` (static buffers).

        ``observations``: ``(batch, M)`` indices or a list of M ``(batch,)``
        arrays; ``empirical_prior``: a list of F ``(batch, S_f)`` arrays or
        one flat ``(batch, sum S)`` tensor. Omitted inputs keep the buffers'
        contents."""
        self.load(observations, empirical_prior)
        for g in self.graphs:
            g.replay()
        return self.qs, self.q_pi, self.G, self.action

    def load(self, observations=None, empirical_prior=None):
        """Copy new inputs into the static buffers on the current stream
        (asynchronous from pinned host memory); omitted inputs are kept."""
        if observations is not None:
            if isinstance(observations, (list, tuple)):
                obs = torch.stack([torch.as_tensor(x).reshape(-1) for x in observations], dim=-1)
            else:
                obs = torch.as_tensor(observations)
            self.obs.copy_(obs.reshape(self.obs.shape), non_blocking=True)
        if empirical_prior is not None:
            if isinstance(empirical_prior, (list, tuple)):
                o = self.agent._qs_offsets
                for f, p in enumerate(empirical_prior):
                    self.prior[:, o[f]:o[f + 1]].copy_(torch.as_tensor(p).reshape(-1, o[f + 1] - o[f]),
                                                       non_blocking=True)
            else:
                self.prior.copy_(torch.as_tensor(empirical_prior).reshape(self.prior.shape), non_blocking=True)


class PipelinedAgentStep:
    """Successive agent steps from host buffers with the copies off the
    compute stream: two ``GraphedAgentStep`` buffer sets, used by steps k and
    k + 1 in turn. Step k copies its observations and prior from host memory
    into set k % 2 on an input stream, which waits only until step k - 2 has
    finished with that set. It then replays the set's graphs on the current
    stream once the copy has landed, and copies the action back on an output
    stream. So the input copy of step k + 1 and the output copy of step k run
    while the GPU computes. Every step still makes both copies. ``step``
    returns the set's static outputs, which step k + 2 overwrites.
    Deterministic action selection only (as ``GraphedAgentStep``). Host
    inputs are read by an asynchronous copy: they must not change until the
    step's outputs are ready.

    ``begin(event)`` makes the copy streams wait for ``event`` (recorded on
    the compute stream, e.g. the start of a timed region), and ``drain()``
    makes the current stream wait for every copy issued so far, so that an
    event recorded after it covers them."""

    def __init__(self, agent: Agent, warmup: int = 2):
        dev = agent.device
        self.sets = [GraphedAgentStep(agent, warmup) for _ in range(2)]
        self.in_stream, self.out_stream = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        self._in_ready = [torch.cuda.Event() for _ in range(2)]  # inputs of the set's current step landed
        self._done = [torch.cuda.Event() for _ in range(2)]      # the set's step computed: inputs free, outputs ready
        self._out_done = [torch.cuda.Event() for _ in range(2)]  # the set's action copied out: action buffer free
        self._k = 0

    def begin(self, event: torch.cuda.Event) -> None:
        self.in_stream.wait_event(event)
        self.out_stream.wait_event(event)

    def step(self, observations, empirical_prior, action_out: torch.Tensor | None = None):
        """One step from host (pinned) or device inputs: ``observations``
        ``(batch, M)``, ``empirical_prior`` flat ``(batch, sum S)`` or a list
        of F ``(batch, S_f)`` arrays. With ``action_out`` (a pinned
        ``(batch, F)`` int32 host tensor) the action is copied into it.
        Returns ``(qs, q_pi, G, action)`` of this step's buffer set."""
        if observations is None or empirical_prior is None:
            # the buffer set was last filled two steps back: there is no previous input to keep
            raise ValueError("PipelinedAgentStep.step needs both observations and empirical_prior")
        i = self._k & 1
        s = self.sets[i]
        comp = torch.cuda.current_stream(s.obs.device)
        parts = list(empirical_prior) if isinstance(empirical_prior, (list, tuple)) else [empirical_prior]
        parts += list(observations) if isinstance(observations, (list, tuple)) else [observations]
        dev_parts = [x for x in parts if isinstance(x, torch.Tensor) and x.is_cuda]
        if dev_parts:
            self.in_stream.wait_stream(comp)  # device inputs may still be in the making on the compute stream
            for x in dev_parts:
                x.record_stream(self.in_stream)  # and their memory stays theirs until the copy has read it
        with torch.cuda.stream(self.in_stream):
            self.in_stream.wait_event(self._done[i])  # step k - 2 has read this set's inputs
            s.load(observations, empirical_prior)
            self._in_ready[i].record(self.in_stream)
        comp.wait_event(self._in_ready[i])
        comp.wait_event(self._out_done[i])  # step k - 2's action has left this set's buffer
        for g in s.graphs:
            g.replay()
        self._done[i].record(comp)
        if action_out is not None:
            with torch.cuda.stream(self.out_stream):
                self.out_stream.wait_event(self._done[i])
                action_out.copy_(s.action, non_blocking=True)
                self._out_done[i].record(self.out_stream)
        self._k += 1
        return s.qs, s.q_pi, s.G, s.action

    def drain(self) -> None:
        comp = torch.cuda.current_stream(self.sets[0].obs.device)
        comp.wait_stream(self.in_stream)
        comp.wait_stream(self.out_stream)

