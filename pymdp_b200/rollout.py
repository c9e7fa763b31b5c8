"""Closed-loop rollout of thousands of agents of uneven sizes in one launch.

The reference runs ``rollout`` (``pymdp/envs/rollout.py:468-700``) as a
``lax.scan`` over ``infer_and_plan`` (``:370-466``) and ``env.step``
(``pymdp/envs/env.py:352-378``), vmapped over a batch whose agents must all
share one shape. :class:`UnevenRollout` takes agents whose factor, modality,
observation and policy counts all differ, packs them into one set of device
buffers with a per-agent descriptor (``b2_ro_agent``), cuts every agent's
policy set into tiles (``b2_ro_tile``, sorted largest first) and runs all
steps in ONE cooperative persistent launch (``b2_rollout``) that a CUDA
graph can hold (:meth:`UnevenRollout.capture`). :func:`autotune` picks the
launch shape (threads per CTA, K chunk, tile width) by timing candidates on
the batch itself.

Semantics per agent (``inference_algo="fpi"``, no learning, deterministic
action selection, each agent's environment built from its own A / B / D):
the first prior is D, later ones ``B[..., a_prev] . qs_prev``; FPI in FP64;
neg-EFE (utility + state information gain) over all ``prod(U)^T`` policies;
``q_pi = softmax(gamma G + log E)`` with E uniform; the action is the first
step of the first maximum of ``q_pi``; the environment then draws the next
state from ``B[:, s, a]`` and the observation from ``A[:, s']`` with a
counter-based generator (SplitMix64 over seed, agent, step and stream).
"""

from __future__ import annotations

import ctypes
import hashlib
import json
import os
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np
import torch

from . import _lib
from ._lib import RoAgent, RoBuffers, RoConfig, RoTile, check

PRECISION = {"fp32": _lib.PRECISIONS["fp32"], "bf16": _lib.PRECISIONS["bf16"]}
SYNC_EXTRA = 32


@dataclass
class AgentSpec:
    """One agent: ``A[m]`` ``(O_m, *S[deps_m])`` with ``deps_m`` ascending,
    ``B[f]`` ``(S_f, S_f, U_f)`` (factor-local), ``C[m]`` ``(O_m,)``,
    ``D[f]`` ``(S_f,)``."""

    A: list
    B: list
    C: list
    D: list
    A_dependencies: list
    policy_len: int
    gamma: float = 16.0
    S: list = field(init=False)
    O: list = field(init=False)
    U: list = field(init=False)

    def __post_init__(self):
        self.A = [np.ascontiguousarray(a, np.float32) for a in self.A]
        self.B = [np.ascontiguousarray(b, np.float32) for b in self.B]
        self.C = [np.ascontiguousarray(c, np.float32).reshape(-1) for c in self.C]
        self.D = [np.ascontiguousarray(d, np.float32).reshape(-1) for d in self.D]
        self.A_dependencies = [[int(x) for x in d] for d in self.A_dependencies]
        self.S = [int(b.shape[0]) for b in self.B]
        self.U = [int(b.shape[2]) for b in self.B]
        self.O = [int(a.shape[0]) for a in self.A]
        for m, (a, deps) in enumerate(zip(self.A, self.A_dependencies)):
            if list(deps) != sorted(set(deps)):
                raise ValueError(f"A_dependencies[{m}] must be strictly ascending")
            if tuple(a.shape[1:]) != tuple(self.S[d] for d in deps):
                raise ValueError(f"A[{m}] shape {a.shape} does not match its dependencies")
        for f, b in enumerate(self.B):
            if b.ndim != 3 or b.shape[0] != b.shape[1]:
                raise ValueError(f"B[{f}] must be (S_f, S_f, U_f)")

    @property
    def num_policies(self) -> int:
        return int(np.prod(self.U)) ** int(self.policy_len)

    @property
    def observed(self) -> list:
        """Factors some modality depends on."""
        return sorted({d for deps in self.A_dependencies for d in deps})

    @property
    def num_reduced_policies(self) -> int:
        """Policies over the observed factors' actions only (unobserved
        factors leave neg-EFE unchanged)."""
        return int(np.prod([self.U[f] for f in self.observed])) ** int(self.policy_len)


def make_uneven_agents(n_agents: int = 2000, seed: int = 0, k_cap: int = 4096, p_cap: int = 256,
                       gamma: float = 16.0, max_factors: int = 4, max_states: int = 64, max_modalities: int = 6,
                       max_obs: int = 32, max_policy_len: int = 4) -> list[AgentSpec]:
    """The uneven-size workload: per agent F ~ U{1..4} factors of S_f ~
    U{2..64} states with U_f ~ U{1..min(4, S_f)} controls, M ~ U{1..6}
    modalities of O_m ~ U{2..32} observations on a random non-empty factor
    subset (redrawn while prod S over it exceeds ``k_cap``), policy_len ~
    U{1..4} (lowered while prod(U)^T exceeds ``p_cap``), A and every B column
    ~ Dirichlet(0.5), C ~ N(0, 1), D uniform. The ``max_*`` arguments shrink
    the ranges (for small test batches)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_agents):
        F = int(rng.integers(1, max_factors + 1))
        S = [int(x) for x in rng.integers(2, max_states + 1, size=F)]
        U = [int(rng.integers(1, min(4, s) + 1)) for s in S]
        M = int(rng.integers(1, max_modalities + 1))
        O = [int(x) for x in rng.integers(2, max_obs + 1, size=M)]
        deps = []
        for _m in range(M):
            while True:
                k = int(rng.integers(1, F + 1))
                d = sorted(int(x) for x in rng.choice(F, k, replace=False))
                if int(np.prod([S[i] for i in d])) <= k_cap:
                    break
            deps.append(d)
        T = int(rng.integers(1, max_policy_len + 1))
        while int(np.prod(U)) ** T > p_cap and T > 1:
            T -= 1
        A = []
        for o, d in zip(O, deps):
            g = rng.gamma(0.5, size=(o, int(np.prod([S[i] for i in d]))))
            A.append((g / g.sum(0, keepdims=True)).astype(np.float32).reshape((o,) + tuple(S[i] for i in d)))
        B = []
        for s, u in zip(S, U):
            g = rng.gamma(0.5, size=(s, s, u))
            B.append((g / g.sum(0, keepdims=True)).astype(np.float32))
        C = [rng.normal(size=o).astype(np.float32) for o in O]
        D = [np.full(s, 1.0 / s, np.float32) for s in S]
        out.append(AgentSpec(A, B, C, D, deps, T, gamma))
    return out


def _descriptor(spec: AgentSpec, offs: dict) -> RoAgent:
    g = RoAgent()
    F, M = len(spec.S), len(spec.O)
    if not (1 <= F <= _lib.RO_MAX_F and 1 <= M <= _lib.RO_MAX_M):
        raise NotImplementedError(f"rollout supports 1..{_lib.RO_MAX_F} factors and 1..{_lib.RO_MAX_M} modalities")
    g.F, g.M, g.T = F, M, int(spec.policy_len)
    nu = int(np.prod(spec.U))
    g.n_multi, g.P, g.w0 = nu, nu ** g.T, nu ** (g.T - 1)
    g.S_tot = int(sum(spec.S))
    qoff = np.cumsum([0] + spec.S)
    for f in range(F):
        g.S[f], g.U[f], g.qs_off[f] = spec.S[f], spec.U[f], int(qoff[f])
        g.ustride[f] = int(np.prod(spec.U[f + 1:]))
    obs = set(spec.observed)
    nr = 1
    for f in range(F - 1, -1, -1):
        g.ustride_r[f] = nr if f in obs else 0
        nr *= spec.U[f] if f in obs else 1
    g.obs_mask = sum(1 << f for f in obs)
    g.n_multi_r, g.P_r, g.w0_r = nr, nr ** g.T, nr ** (g.T - 1)
    sumK = 0
    for m, deps in enumerate(spec.A_dependencies):
        K = int(np.prod([spec.S[d] for d in deps]))
        g.O[m], g.K[m], g.rank[m] = spec.O[m], K, len(deps)
        stride = 1
        for j in range(len(deps) - 1, -1, -1):
            g.dep[m][j] = deps[j]
            g.dstride[m][j] = stride
            stride *= spec.S[deps[j]]
        g.A_off[m], g.C_off[m] = offs["A"][m], offs["C"][m]
        sumK += K
    g.sum_K = sumK
    for f in range(F):
        g.B_off[f] = offs["B"][f]
    g.D_off, g.ll_off, g.qs_base, g.G_off = offs["D"], offs["ll"], offs["qs"], offs["G"]
    g.gamma = float(spec.gamma)
    return g


def tile_cost(spec: AgentSpec, p_lo: int, p_hi: int) -> float:
    """Multiply-adds of one tile of reduced policies: per depth, its distinct
    prefixes times the contraction rows x K plus the B roll-out of the
    observed factors."""
    nu = int(np.prod([spec.U[f] for f in spec.observed]))
    per_col = (sum((o + 1) * int(a[0].size) for o, a in zip(spec.O, spec.A))
               + sum(spec.S[f] ** 2 for f in spec.observed))
    cost, W = 0.0, nu ** (spec.policy_len - 1)
    for _t in range(spec.policy_len):
        cost += ((p_hi - 1) // W + 1 - p_lo // W) * per_col
        W = max(W // nu, 1)
    return cost


def make_tiles(specs: Sequence[AgentSpec], cols: int, balance_tiles: int | None = None) -> np.ndarray:
    """Cut each agent's reduced policies into tiles of at most ``cols``
    policies (with round_up(width, 8) x S_tot within the shared-memory
    prefix table), largest cost first. With ``balance_tiles``, an agent whose
    policies cost more than (total cost / balance_tiles) per tile gets
    narrower tiles, so no tile dominates a step (off by default: on the
    2000-agent workload, balancing to 1776 tiles cut the costliest tile 5x but
    made the rollout 25% slower, as narrow tiles share fewer prefixes and
    carry more fixed cost). Returns ``(n_tiles, 4)`` int32 rows
    ``(agent, p_lo, p_hi, 0)``."""
    target = None
    if balance_tiles:
        total = sum(tile_cost(sp, 0, sp.num_reduced_policies) for sp in specs)
        target = total / float(balance_tiles)
    rows, costs = [], []
    for i, sp in enumerate(specs):
        P, St = sp.num_reduced_policies, int(sum(sp.S))
        width = max(1, min(int(cols), P, _lib.RO_TAB_FLOATS // St // 8 * 8))
        if target is not None:
            per_policy = tile_cost(sp, 0, P) / P
            width = max(1, min(width, int(target // max(per_policy, 1e-9))))
        for lo in range(0, P, width):
            hi = min(P, lo + width)
            rows.append((i, lo, hi, 0))
            costs.append(tile_cost(sp, lo, hi))
    order = np.argsort(-np.asarray(costs), kind="stable")
    return np.asarray(rows, dtype=np.int32)[order]


def _signature(specs: Sequence[AgentSpec]) -> str:
    h = hashlib.sha1()
    for sp in specs:
        h.update(np.asarray(sp.S + [-1] + sp.O + [-1] + sp.U + [sp.policy_len], np.int64).tobytes())
        for d in sp.A_dependencies:
            h.update(np.asarray(d + [-2], np.int64).tobytes())
    return h.hexdigest()[:16]


class UnevenRollout:
    """Device-resident batch of uneven agents and their environments."""

    def __init__(self, agents: Sequence[AgentSpec], *, precision: str = "fp32", num_iter: int = 16,
                 use_utility: bool = True, use_states_info_gain: bool = True, device="cuda", threads: int = 256,
                 kc: int = 64, cols: int = 32):
        if precision not in PRECISION:
            raise ValueError(f"precision must be one of {sorted(PRECISION)}")
        self.specs = list(agents)
        self.n = len(self.specs)
        if self.n == 0:
            raise ValueError("no agents")
        self.precision, self.num_iter = precision, int(num_iter)
        self.flags = (_lib.FLAG_USE_UTILITY if use_utility else 0) | (
            _lib.FLAG_USE_STATES_INFO_GAIN if use_states_info_gain else 0)
        self.device = torch.device(device)
        self.signature = _signature(self.specs)
        self._pack_host()
        self._upload()
        self.config = RoConfig(int(threads), int(kc), int(cols), PRECISION[precision])
        self._bufs = None
        self._steps = 0
        self._records = None
        self.set_tiles(int(cols))
        self._setup()

    # --------------------------------------------------------------- packing
    def _pack_host(self):
        A_parts, B_parts, C_parts, D_parts = [], [], [], []
        descs = (RoAgent * self.n)()
        nA = nB = nC = nD = nll = nqs = nG = 0
        for i, sp in enumerate(self.specs):
            offs = {"A": [], "C": [], "B": []}
            for a, c in zip(sp.A, sp.C):
                O, K = a.shape[0], int(a[0].size)
                blk = np.zeros((O + 1, K), np.float32)
                blk[:O] = a.reshape(O, K)
                offs["A"].append(nA)
                A_parts.append(blk.reshape(-1))
                nA += blk.size
                offs["C"].append(nC)
                C_parts.append(c)
                nC += c.size
            for b in sp.B:
                offs["B"].append(nB)
                # stored action-major: [u][prev][next], so a transition column and
                # a roll-out row are contiguous
                B_parts.append(np.ascontiguousarray(b.transpose(2, 1, 0)).reshape(-1))
                nB += b.size
            offs["D"] = nD
            D_parts.append(np.concatenate(sp.D))
            nD += sum(sp.S)
            offs["ll"] = nll
            nll += sum(int(a[0].size) for a in sp.A)
            offs["qs"] = nqs
            nqs += sum(sp.S)
            offs["G"] = nG
            nG += sp.num_policies
            descs[i] = _descriptor(sp, offs)
        self.descs = descs
        self.host = {"Aprime": np.concatenate(A_parts), "B": np.concatenate(B_parts), "C": np.concatenate(C_parts),
                     "D": np.concatenate(D_parts)}
        self.counts = {"ll": nll, "qs": nqs, "G": nG}

    def _upload(self):
        dev = self.device
        t = {k: torch.as_tensor(v, device=dev) for k, v in self.host.items()}
        t["Aprime_bf16"] = (torch.empty(t["Aprime"].numel(), dtype=torch.int16, device=dev)
                            if self.precision == "bf16" else None)
        t["ll"] = torch.empty(max(self.counts["ll"], 1), dtype=torch.float64, device=dev)
        t["qs"] = torch.empty(self.counts["qs"], dtype=torch.float32, device=dev)
        t["qs64"] = torch.empty(self.counts["qs"], dtype=torch.float64, device=dev)
        t["G"] = torch.empty(self.counts["G"], dtype=torch.float32, device=dev)
        t["env_state"] = torch.zeros((self.n, _lib.RO_MAX_F), dtype=torch.int32, device=dev)
        t["obs"] = torch.zeros((self.n, _lib.RO_MAX_M), dtype=torch.int32, device=dev)
        raw = ctypes.string_at(ctypes.addressof(self.descs), ctypes.sizeof(self.descs))
        t["agents"] = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(dev)
        self.t = t

    def set_tiles(self, cols: int):
        """Re-cut the policy tiles for tile width ``cols``."""
        self.tiles_np = np.ascontiguousarray(make_tiles(self.specs, cols))
        self.tiles_host = (RoTile * len(self.tiles_np))()
        ctypes.memmove(self.tiles_host, self.tiles_np.ctypes.data, self.tiles_np.nbytes)
        self.t["tiles"] = torch.as_tensor(self.tiles_np.reshape(-1), device=self.device)
        self.config.cols = int(cols)
        self._bufs = None

    def _buffers(self, steps: int, record: bool) -> RoBuffers:
        if self._steps < steps or "sync" not in self.t:
            self.t["sync"] = torch.zeros(2 * steps + SYNC_EXTRA, dtype=torch.int32, device=self.device)
            self._steps = steps
            self._bufs = None
        if record and (self._records is None or self._records["steps"] != steps):
            dev = self.device
            self._records = {
                "steps": steps,
                "obs": torch.zeros((steps, self.n, _lib.RO_MAX_M), dtype=torch.int16, device=dev),
                "state": torch.zeros((steps, self.n, _lib.RO_MAX_F), dtype=torch.int16, device=dev),
                "action": torch.zeros((steps, self.n, _lib.RO_MAX_F), dtype=torch.int16, device=dev),
                "qs": torch.zeros((steps, self.counts["qs"]), dtype=torch.float32, device=dev),
                "G": torch.zeros((steps, self.counts["G"]), dtype=torch.float32, device=dev),
            }
            self._bufs = None
        if self._bufs is not None and self._bufs_record == record:
            return self._bufs
        t = self.t
        p = lambda x: 0 if x is None else x.data_ptr()  # noqa: E731
        rec = self._records if record else None
        b = RoBuffers(p(t["agents"]), p(t["tiles"]), p(t["Aprime"]), p(t["Aprime_bf16"]), t["Aprime"].numel(),
                      p(t["B"]), t["B"].numel(), p(t["C"]), t["C"].numel(), p(t["D"]), t["D"].numel(), p(t["ll"]),
                      t["ll"].numel(), p(t["qs"]), p(t["qs64"]), t["qs"].numel(), p(t["G"]), t["G"].numel(),
                      p(t["env_state"]), p(t["obs"]), p(rec and rec["obs"]), p(rec and rec["state"]),
                      p(rec and rec["action"]), p(rec and rec["qs"]), p(rec and rec["G"]), p(t["sync"]),
                      t["sync"].numel())
        self._bufs, self._bufs_record = b, record
        return b

    def _setup(self):
        b = self._buffers(1, False)
        check(_lib.load().b2_rollout_setup(self._stream(), ctypes.addressof(self.descs), self.n, ctypes.byref(b),
                                           self.flags))

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    # ----------------------------------------------------------------- running
    def run(self, steps: int, seed: int = 0, record: bool = False):
        """Launch a ``steps``-step rollout from an environment reset on the
        current stream (asynchronous). With ``record`` the per-step
        observations, states, actions, posteriors and neg-EFE are kept (see
        :meth:`records`)."""
        b = self._buffers(int(steps), record)
        check(_lib.load().b2_rollout(self._stream(), ctypes.addressof(self.descs), self.n,
                                     ctypes.addressof(self.tiles_host), len(self.tiles_np), ctypes.byref(b),
                                     int(steps), int(seed) & ((1 << 64) - 1), self.num_iter, self.flags,
                                     ctypes.byref(self.config)))

    def check_status(self):
        """Raise if the last rollout aborted on the device (reads 2 words)."""
        st = self.t["sync"][2:4].cpu().tolist()
        if st[0]:
            raise RuntimeError(f"rollout aborted on the device (code {st[1]}: grid barrier wait expired)")

    def records(self) -> list:
        """Host copies of the recorded trajectory, per agent: ``obs[t][m]``,
        ``state[t][f]``, ``action[t][f]``, ``qs[t]`` (list per factor) and
        ``G[t]``."""
        if self._records is None:
            raise RuntimeError("run(..., record=True) first")
        r = {k: v.cpu().numpy() for k, v in self._records.items() if k != "steps"}
        out = []
        for i, sp in enumerate(self.specs):
            g = self.descs[i]
            qoff = np.cumsum([0] + sp.S)
            qs = r["qs"][:, g.qs_base:g.qs_base + g.S_tot]
            out.append({"obs": r["obs"][:, i, :len(sp.O)].astype(np.int64),
                        "state": r["state"][:, i, :len(sp.S)].astype(np.int64),
                        "action": r["action"][:, i, :len(sp.S)].astype(np.int64),
                        "qs": [[qs[t, qoff[f]:qoff[f + 1]] for f in range(len(sp.S))] for t in range(qs.shape[0])],
                        "G": r["G"][:, g.G_off:g.G_off + g.P]})
        return out

    def capture(self, steps: int, seed: int = 0, record: bool = False) -> torch.cuda.CUDAGraph:
        """Capture one ``steps``-step rollout (sync reset + the persistent
        launch) in a CUDA graph; ``graph.replay()`` re-runs it from the reset."""
        self.run(steps, seed, record)  # validates and allocates outside the capture
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run(steps, seed, record)
        return g


# --------------------------------------------------------------- autotuner
CANDIDATES = [(t, kc, c) for t in (128, 256, 512) for kc in (32, 64) for c in (16, 32, 64)]
_TUNE_CACHE: dict = {}


def autotune(ro: UnevenRollout, steps: int = 2, candidates=None, cache_path: str | None = None, repeats: int = 2):
    """Time every (threads, kc, cols) candidate on ``ro`` itself (``steps``
    rollout steps, best of ``repeats`` after one warm-up) and keep the
    fastest in ``ro.config``. Results are cached per (device, precision,
    agent-shape signature, num_iter) in memory and, with ``cache_path``, in a
    JSON file. Returns ``(best, timings)`` with timings in ms."""
    dev_name = torch.cuda.get_device_name(ro.device)
    key = f"{dev_name}|{ro.precision}|{ro.signature}|{ro.num_iter}|{ro.n}"
    disk = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as fh:
            disk = json.load(fh)
    hit = _TUNE_CACHE.get(key) or disk.get(key)
    if hit is not None:
        _apply(ro, hit["best"])
        return tuple(hit["best"]), hit["timings"]
    timings = {}
    for cand in (candidates or CANDIDATES):
        _apply(ro, cand)
        ro.run(steps)
        best = None
        for _ in range(repeats):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ro.run(steps)
            e1.record()
            torch.cuda.synchronize(ro.device)
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        ro.check_status()
        timings[",".join(map(str, cand))] = best
    best_key = min(timings, key=timings.get)
    best = tuple(int(x) for x in best_key.split(","))
    _apply(ro, best)
    entry = {"best": list(best), "timings": timings}
    _TUNE_CACHE[key] = entry
    if cache_path:
        disk[key] = entry
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as fh:
            json.dump(disk, fh, indent=1)
    return best, timings


def _apply(ro: UnevenRollout, cand):
    threads, kc, cols = (int(x) for x in cand)
    ro.config.threads, ro.config.kc = threads, kc
    if cols != ro.config.cols:
        ro.set_tiles(cols)
