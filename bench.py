"""Benchmark: agent-steps/s of the FPI + EFE agent step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one "step" = one agent step for every agent of the batch):
the EFE benchmark model — 256 agents, num_states [32, 16, 8],
num_controls [4, 4, 1], policy_len 3 (4096 policies), 5 modalities with
num_obs [16, 16, 8, 8, 4] depending on all factors, A ~ Dirichlet(0.5),
B ~ Dirichlet(0.5) per action slice, C ~ N(0, 1), E uniform, gamma 16 —
running infer_states (fused FPI, 16 iterations, one-hot observations) ->
infer_policies (neg-EFE of all policies + q_pi) -> sample_action
(deterministic). Synthetic seeded inputs with those shapes/distributions.

* ``value``: device time (CUDA events, max over ranks) with every input
  resident in HBM, the whole step replayed as one CUDA graph
  (``Agent.capture_step``); L2 is flushed (a 256 MiB write) between timed
  steps, outside the per-step event pairs.
* ``e2e``: the same step through the public API
  (``Agent.capture_pipeline().step``) with host buffers: every step copies
  pinned observations + priors in and its actions out, on copy streams
  beside the neighbouring steps' compute, all inside the timed region.
* ``roofline``: the dominant launch (the factored neg-EFE + q_pi), its
  algorithmic HBM bytes per agent over its event-timed duration inside the
  timed steps (tensor-pipe FLOPs for ``--efe dense``).
* ``cpu_baseline``: the reference's own CPU kernels (NegEfeCpu + FpiCpu,
  compiled from its sources into ``oracle/_ref``) on the host cores for a
  bounded sample of the same agents; the FP64 oracle on another sample
  gives ``error_vs_fp64``, the GPU outputs' max error against FP64.
* ``--impl reference``: the same reference CPU step alone, as the
  reference arm.

Multi-GPU: agents are independent, so each rank runs its own 256 agents
(weak scaling, no data-path collective); the only collective is the
max-over-ranks of the timing.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

S = [32, 16, 8]
O = [16, 16, 8, 8, 4]
U = [4, 4, 1]
T = 3
AGENTS = 256
NUM_ITER = 16
GAMMA = 16.0


def workload(agents: int) -> str:
    return (f"agent step (FPI 16 iters + EFE all 4096 policies + action), {agents} agents, S=[32,16,8], "
            "O=[16,16,8,8,4], U=[4,4,1], policy_len=3")


def make_model(seed: int, agents: int):
    rng = np.random.default_rng(seed)

    def dirc(shape, alpha):
        g = rng.gamma(alpha, size=shape) + 1e-30
        return (g / g.sum(1, keepdims=True)).astype(np.float32)

    F, M = len(S), len(O)
    A = [dirc((agents, O[m]) + tuple(S), 0.5) for m in range(M)]
    B = [dirc((agents, S[f], S[f], U[f]), 0.5) for f in range(F)]
    C = [rng.normal(size=(agents, o)).astype(np.float32) for o in O]
    D = [dirc((agents, s), 1.0) for s in S]
    obs = rng.integers(0, np.array(O), size=(agents, M)).astype(np.int32)
    return A, B, C, D, obs


# FPI-only benchmark model: 4096 agents, 4 factors x 16 states, 6 modalities x
# 32 observations, each A_m on 2 randomly chosen factors (K = 256), A columns
# ~ Dirichlet(0.5), D ~ Dirichlet(1), random observations, 16 iterations.
FPI_AGENTS, FPI_S, FPI_O, FPI_ITERS = 4096, [16] * 4, [32] * 6, 16


def fpi_bytes_per_agent_cfg(S, O, deps) -> float:
    """Algorithmic HBM bytes of one fused FPI agent: the observed A slices, the
    prior in, the posterior out and the observation indices."""
    K = [int(np.prod([S[d] for d in dp])) for dp in deps]
    return 4.0 * sum(K) + 8.0 * sum(S) + 4.0 * len(O)


def run_fpi_config(dev, steps: int, warmup: int, flush, agents: int = FPI_AGENTS):
    """FPI alone on the FPI benchmark model (4096 agents; more for the
    throughput sweep): device time per launch (L2 flushed before each),
    agent-steps/s and algorithmic HBM GB/s."""
    import torch

    from pymdp_b200 import ffi

    rng = np.random.default_rng(2)
    deps = [sorted(rng.choice(len(FPI_S), 2, replace=False).tolist()) for _ in FPI_O]
    gen = torch.Generator(device=dev).manual_seed(2)

    def dirichlet(shape, alpha):
        g = torch._standard_gamma(torch.full(shape, alpha, device=dev), generator=gen) + 1e-30
        return g / g.sum(1, keepdim=True)

    A = [dirichlet((agents, o) + tuple(FPI_S[d] for d in dp), 0.5) for o, dp in zip(FPI_O, deps)]
    A_flat, A_off = ffi.flatten_ragged_f32(A, 1, dev)
    del A
    prior = torch.cat([dirichlet((agents, s), 1.0) for s in FPI_S], dim=1).contiguous()
    obs = torch.stack([torch.randint(0, o, (agents,), device=dev, generator=gen) for o in FPI_O],
                      dim=1).to(torch.int32).contiguous()
    out = torch.empty_like(prior)

    def launch():
        ffi.fpi_obs_flat(A_flat, int(A_off[-1]), A_off, FPI_O, obs, prior, FPI_S, deps, FPI_ITERS, out=out)

    for _ in range(warmup):
        launch()
    torch.cuda.synchronize(dev)
    evs = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launch()
        e1.record()
        evs.append((e0, e1))
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in evs) / steps
    nbytes = fpi_bytes_per_agent_cfg(FPI_S, FPI_O, deps) * agents
    return {"workload": f"FPI only, {agents} agents, S={FPI_S}, O={FPI_O}, A_m on 2 random factors (K=256), "
                        f"{FPI_ITERS} iterations, L2 flushed before each launch",
            "agent_steps_per_s": agents / (ms * 1e-3), "ms_per_launch": ms,
            "bytes_per_launch": nbytes, "gbs": nbytes / (ms * 1e-3) / 1e9}


LEARN_AGENTS = 256


def learn_bytes_per_agent(S, O, U, A_deps, B_deps) -> float:
    """Algorithmic HBM bytes of one online learning step of one agent (T = 1
    observation, one transition): every pA / pB element read and every A / B
    element written; pA written in the observed row of each column, pB in the
    taken action's slice; beliefs, observations and actions in."""
    KA = [int(np.prod([S[d] for d in dp])) for dp in A_deps]
    KB = [int(np.prod([S[d] for d in dp])) for dp in B_deps]
    a = 8.0 * sum(o * k for o, k in zip(O, KA)) + 4.0 * sum(KA)
    b = 8.0 * sum(s * k * u for s, k, u in zip(S, KB, U)) + 4.0 * sum(s * k for s, k in zip(S, KB))
    return a + b + 4.0 * (2 * sum(S) + len(O) + len(S) + 2)


def run_learn_config(dev, steps: int, warmup: int, flush):
    """Online Dirichlet learning (pA -> A and pB -> B, one observation and one
    transition per agent) on the 256-agent benchmark model: device time per
    step (both launches; L2 flushed before each), agent-steps/s and
    algorithmic HBM GB/s."""
    import torch

    from pymdp_b200 import ffi

    S, O, U = [32, 16, 8], [16, 16, 8, 8, 4], [4, 4, 1]
    A_deps, B_deps = [[0, 1, 2]] * 5, [[0], [1], [2]]
    Bn = LEARN_AGENTS
    lay = ffi.EfeLayout(S, O, U, 1, A_deps, B_deps)
    g = torch.Generator(device=dev).manual_seed(7)
    pA = torch.rand((Bn, int(lay.A_offsets[-1])), device=dev, generator=g) + 0.5
    pB = torch.rand((Bn, int(lay.B_offsets[-1])), device=dev, generator=g) + 0.5
    A, Bm = torch.empty_like(pA), torch.empty_like(pB)
    q = torch.cat([torch.softmax(torch.randn((Bn, 2, s), device=dev, generator=g) * 3, -1) for s in S], -1)
    q1 = q[:, 1:].contiguous()
    obs = torch.stack([torch.randint(0, o, (Bn, 1), device=dev, generator=g) for o in O], -1).to(torch.int32)
    act = torch.stack([torch.randint(0, u, (Bn, 1), device=dev, generator=g) for u in U], -1).to(torch.int32)
    obs, act = obs.contiguous(), act.contiguous()
    lr = torch.full((Bn,), 1e-3, device=dev)
    work = torch.zeros(1, dtype=torch.int32, device=dev)

    def launch():
        lay.learn_A(pA, A, obs, q1, lr, Bn, 1)
        lay.learn_B(pB, Bm, q, act, lr, work, Bn, 2)

    for _ in range(warmup):
        launch()
    torch.cuda.synchronize(dev)
    evs = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launch()
        e1.record()
        evs.append((e0, e1))
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in evs) / steps
    nbytes = learn_bytes_per_agent(S, O, U, A_deps, B_deps) * Bn
    return {"workload": f"online Dirichlet learning of A and B, {Bn} agents, S={S}, O={O}, U={U}, every modality "
                        f"on every factor, 1 observation + 1 transition per agent, L2 flushed before each step",
            "agent_steps_per_s": Bn / (ms * 1e-3), "ms_per_step": ms, "launches_per_step": 3,
            "bytes_per_step": nbytes, "gbs": nbytes / (ms * 1e-3) / 1e9}


HMM_AGENTS, HMM_T, HMM_K, HMM_U, HMM_O = 4096, 64, 32, 4, [16, 8]


def hmm_bytes_per_agent(T, K, U, O) -> float:
    """Algorithmic HBM bytes of one agent's exact filter + smoother: A, B,
    prior, observations and actions in; mll, filtered, predicted, smoothed
    and the pairwise posteriors (joint and conditional) out."""
    ins = 4.0 * (sum(O) * K + K * K * U + K + T * len(O) + (T - 1))
    outs = 4.0 * (1 + 3 * T * K + 2 * (T - 1) * K * K)
    return ins + outs


def run_hmm_config(dev, steps: int, warmup: int, flush, agents: int = HMM_AGENTS):
    """Exact single-factor HMM filtering + smoothing (run_exact_single_factor_hmm_scan
    with the joint posteriors) for 4096 agents: device time per launch (L2
    flushed before each), agent-sequences/s and algorithmic HBM GB/s."""
    import torch

    from pymdp_b200 import hmm

    Bn, T, K, U, O = agents, HMM_T, HMM_K, HMM_U, HMM_O
    g = torch.Generator(device=dev).manual_seed(11)
    A = [torch.softmax(torch.randn((Bn, o, K), device=dev, generator=g) * 2, dim=1) for o in O]
    B = torch.softmax(torch.randn((Bn, K, K, U), device=dev, generator=g) * 2, dim=1).contiguous()
    prior = torch.softmax(torch.randn((Bn, K), device=dev, generator=g), dim=1)
    obs = [torch.randint(0, o, (Bn, T), device=dev, generator=g, dtype=torch.int32) for o in O]
    acts = torch.randint(0, U, (Bn, T - 1), device=dev, generator=g, dtype=torch.int32)
    A_flat = torch.cat([a.reshape(Bn, -1) for a in A], dim=-1).contiguous()
    obs_i = torch.stack(obs, dim=-1).contiguous()
    out = hmm.hmm_outputs(Bn, T, K, ("mll", "filtered", "predicted", "smoothed", "joint", "cond"), dev)

    def launch():
        hmm.hmm_smoother_packed(A_flat, 1, O, obs_i, False, prior, B, 1, U, acts, "index", out)

    for _ in range(warmup):
        launch()
    torch.cuda.synchronize(dev)
    evs = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launch()
        e1.record()
        evs.append((e0, e1))
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in evs) / steps
    nbytes = hmm_bytes_per_agent(T, K, U, O) * Bn
    return {"workload": f"exact single-factor HMM filter + smoother, {Bn} agents, T={T}, K={K}, U={U}, O={O}, "
                        f"index observations, all outputs incl. joint and conditional pairwise posteriors, L2 "
                        f"flushed before each launch",
            "agent_sequences_per_s": Bn / (ms * 1e-3), "ms_per_launch": ms, "bytes_per_launch": nbytes,
            "gbs": nbytes / (ms * 1e-3) / 1e9}


SEQ_AGENTS, SEQ_T, SEQ_S, SEQ_O, SEQ_ITERS = 4096, 8, [16, 8], [16, 8], 16


def run_seq_config(dev, steps: int, warmup: int, flush):
    """Sequence inference (run_mmp, pymdp/algos.py:392-430) for 4096 agents:
    a window of 8 steps, S=[16, 8], O=[16, 8] on both factors, factor-local
    action-conditioned transitions, index observations, 16 iterations of
    tau 0.25. Device time per launch (L2 flushed before each) and
    agent-windows/s on inputs packed once (``seq.prepare``), beside the time of
    the list-taking ``seq.run_mmp`` call that packs them every time;
    algorithmic bytes = A, B sequence, observations, prior in and the
    posteriors out."""
    import torch

    from pymdp_b200 import seq

    g = torch.Generator(device=dev).manual_seed(13)
    Bn, T, S, O = SEQ_AGENTS, SEQ_T, SEQ_S, SEQ_O
    K = int(np.prod(S))
    A = [torch.softmax(torch.randn((Bn, o) + tuple(S), device=dev, generator=g) * 2, dim=1) for o in O]
    B = [torch.softmax(torch.randn((Bn, T - 1, s, s), device=dev, generator=g) * 2, dim=2) for s in S]
    obs = [torch.randint(0, o, (Bn, T), device=dev, generator=g, dtype=torch.int32) for o in O]
    prior = [torch.softmax(torch.randn((Bn, s), device=dev, generator=g), dim=1) for s in S]
    deps = [[0, 1]] * len(O)

    def api_call():
        return seq.run_mmp(A, B, obs, prior, deps, [[0], [1]], num_iter=SEQ_ITERS, tau=0.25, distr_obs=False)

    plan = seq.prepare(False, A, B, obs, prior, deps, [[0], [1]], num_iter=SEQ_ITERS, tau=0.25, distr_obs=False)

    def timed(fn):
        for _ in range(max(1, warmup)):
            fn()
        torch.cuda.synchronize(dev)
        evs = []
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            evs.append((e0, e1))
        torch.cuda.synchronize(dev)
        return sum(a.elapsed_time(b) for a, b in evs) / steps

    ms = timed(plan.run)
    ms_api = timed(api_call)
    nbytes = 4.0 * Bn * (sum(O) * K + (T - 1) * sum(s * s for s in S) + T * len(O) + sum(S) + T * sum(S))
    return {"workload": f"run_mmp, {Bn} agents, window T={T}, S={S}, O={O} on both factors, factor-local "
                        f"transitions, index observations, {SEQ_ITERS} iterations (tau 0.25), L2 flushed",
            "agent_windows_per_s": Bn / (ms * 1e-3), "ms_per_launch": ms, "bytes_per_launch": nbytes,
            "gbs": nbytes / (ms * 1e-3) / 1e9,
            "api_ms_per_call": ms_api,
            "api_note": "ms_per_launch: the kernel on inputs packed once (seq.prepare(...).run()); api_ms_per_call: "
                        "seq.run_mmp from the per-modality lists, packing them into flat buffers each call"}


FIT_SUBJECTS, FIT_TRIALS = 1024, 64


def run_fit_config(dev, steps: int, warmup: int, flush):
    """Model fitting: the summed action log-likelihood of 1024 subjects x 64
    trials (S=[8,4], O=[8,4,3] on both factors, U=[4,1], policy_len 2,
    num_iter 16, logits ~ N(0,1), C ~ N(0,1), log gamma ~ N(log 8, 0.3),
    actions sampled from each subject's own model) and its gradient w.r.t.
    every parameter, forward + backward replayed as one CUDA graph. Device
    time per evaluation (L2 flushed before each) and subject-steps/s."""
    import torch

    from pymdp_b200 import _lib
    from pymdp_b200.fitting import FitModel, GraphedLogLikelihood

    fm = FitModel([8, 4], [8, 4, 3], [4, 1], policy_len=2, num_iter=16, device=dev)
    gen = torch.Generator(device=dev).manual_seed(3)
    A, B, C, lg = fm.init_params(FIT_SUBJECTS, gen)
    obs, acts = fm.simulate(A, B, C, lg, FIT_TRIALS, gen)
    params = [x.clone().requires_grad_(True) for x in A + B + C + [lg]]
    n0 = _lib.launch_count()
    graphed = GraphedLogLikelihood(fm, params, obs, acts, warmup=max(warmup, 1))
    native = _lib.launch_count() - n0  # native launches of the warm-up passes plus the captured one
    for _ in range(warmup):
        graphed()
    torch.cuda.synchronize(dev)
    evs = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        graphed()
        e1.record()
        evs.append((e0, e1))
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in evs) / steps
    return {"workload": f"model fitting, {FIT_SUBJECTS} subjects x {FIT_TRIALS} trials, S=[8,4], O=[8,4,3], "
                        "U=[4,1], policy_len 2, num_iter 16: action log-likelihood + gradient w.r.t. A/B logits, "
                        "C and log gamma (native FPI / neg-EFE adjoints, one CUDA graph), L2 flushed before each",
            "subject_steps_per_s": FIT_SUBJECTS * FIT_TRIALS / (ms * 1e-3), "ms_per_evaluation": ms,
            "native_launches_per_evaluation": native // (max(warmup, 1) + 1),
            "log_likelihood": float(graphed.ll.detach())}


RO_AGENTS, RO_STEPS = 2000, 100
FP32_SIMT_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 148 SMs x 128 FP32 lanes x FMA x 1965 MHz


def run_rollout_config(dev, steps: int, warmup: int):
    """Uneven-size closed-loop rollout: 2000 agents of random sizes, 100
    steps of infer_states -> infer_policies -> action -> env step in one
    CUDA-graph-captured persistent launch, launch shape autotuned, for the
    FP32 and BF16 A operand. One replay is one timed step."""
    import torch

    from pymdp_b200.rollout import UnevenRollout, autotune, make_uneven_agents, tile_cost

    specs = make_uneven_agents(RO_AGENTS, seed=0)
    out = {"workload": f"uneven rollout, {RO_AGENTS} agents (F 1-4 of S 2-64, U 1-4, M 1-6 of O 2-32, policy_len "
                       f"1-4, K_m <= 4096, P <= 256), {RO_STEPS} steps per replay of one CUDA graph holding one "
                       "persistent launch; working set (A 237 MB) above L2"}
    for prec in ("fp32", "bf16"):
        ro = UnevenRollout(specs, precision=prec, device=dev)
        best, _ = autotune(ro, steps=2)
        graph = ro.capture(RO_STEPS, seed=1)
        for _ in range(max(warmup, 1)):
            graph.replay()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            graph.replay()
        e1.record()
        torch.cuda.synchronize(dev)
        ro.check_status()
        ms = e0.elapsed_time(e1) / steps
        macs = sum(tile_cost(specs[a], lo, hi) for a, lo, hi, _ in ro.tiles_np) * RO_STEPS
        tf = 2 * macs / (ms * 1e-3) / 1e12
        out[prec] = {"agent_steps_per_s": RO_AGENTS * RO_STEPS / (ms * 1e-3), "ms_per_rollout": ms,
                     "launch_shape": {"threads": best[0], "kc": best[1], "cols": best[2]},
                     "efe_tflops": tf, "roofline": {"bound": "fp32 simt", "achieved": tf,
                                                    "peak": FP32_SIMT_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                                                    "frac": tf / FP32_SIMT_NOMINAL_TFLOPS,
                                                    "peak_source": "nominal"}}
        del graph, ro
    return out


def efe_flops_per_agent(tree: bool = False) -> float:
    """Contraction flops per agent: every policy at every step (dense), or,
    with the policy tree, every distinct prefix once: 2 * sum_t nu^(t+1) *
    sum_m O_m K_m with nu = prod(U)."""
    K = int(np.prod(S))
    nu = int(np.prod(U))
    cols = sum(nu ** (t + 1) for t in range(T)) if tree else T * nu ** T
    return 2.0 * cols * sum(o * K for o in O)


# DRAM bytes per agent of the neg-EFE launch, from ncu captures of 160 agents (A and the per-agent intermediates
# are touched once per agent, so traffic scales with agents): the tensor-core kernel in policy-tree mode; the
# factored launch's history, level-1, tail and combine kernels (dram__bytes_read.sum + dram__bytes_write.sum:
# 3.39 + (136.48 + 29.74) + (54.72 + 0.39) + 5.68 MB; the level-1 intermediates partly spill from L2 and come back
# in the tail).
EFE_TRAFFIC_PER_AGENT = {"tf32x3": (349.50e6 + 9.88e6) / 160,
                         "factored": (3.39e6 + 136.48e6 + 29.74e6 + 54.72e6 + 0.39e6 + 5.68e6) / 160}


def efe_bytes_per_agent() -> float:
    """Algorithmic HBM bytes of one agent's neg-EFE + q_pi on the benchmark
    model: A, B, C (T x O per modality), the beliefs and E read once; G and
    q_pi written once."""
    K = int(np.prod(S))
    P = int(np.prod(U)) ** T
    a = 4.0 * sum(O) * K
    b = 4.0 * sum(s * s * u for s, u in zip(S, U))
    return a + b + 4.0 * (T * sum(O) + sum(S)) + 4.0 * 3 * P


def efe_factored_flops_per_agent() -> float:
    """Multiply-add flops the factored path executes per agent on the
    benchmark model (contraction order: factor 2, then 0, then 1): level 1 over
    A for each depth, level 2 per factor-0 history, level 3 per pair."""
    n = sum(O) + 1
    K = int(np.prod(S))
    total = 0
    for t in range(T):
        h1 = U[0] ** (t + 1)
        h2 = U[1] ** (t + 1)
        total += n * K + h1 * n * S[0] * S[1] + h1 * h2 * n * S[1]
    return 2.0 * total


def fpi_bytes_per_agent() -> float:
    K = int(np.prod(S))
    return 4.0 * len(O) * K + 8.0 * sum(S) + 4.0 * len(O)


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.rows, self._stop = index, [], threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:  # noqa: BLE001
                return
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if "Active" in r[2 + i]
                          and "Not" not in r[2 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _oracle_agent_step(args):
    """One agent's full step with the FP64 oracle: (qs, G, q_pi, action)."""
    from oracle import efe as oefe
    from oracle import fpi as ofpi

    A_b, B_b, C_b, D_b, obs_b = args
    F, M = len(S), len(O)
    A_deps = [list(range(F))] * M
    B_deps = [[f] for f in range(F)]
    pol = oefe.construct_policies(S, U, T)
    E = np.full(len(pol), 1.0 / len(pol))
    o_vec = [np.eye(O[m])[obs_b[m]] for m in range(M)]
    qs = ofpi.run_factorized_fpi([a.astype(np.float64) for a in A_b], o_vec, D_b, A_deps, NUM_ITER)
    q_pi, G = oefe.update_posterior_policies(pol, qs, A_b, B_b, C_b, E, A_deps, B_deps, gamma=GAMMA)
    return qs, G, q_pi, oefe.sample_policy(pol, q_pi)


def _worker_init():
    # one BLAS thread per worker process: the pool supplies the parallelism
    try:
        from threadpoolctl import threadpool_limits

        threadpool_limits(1)
    except Exception:  # noqa: BLE001
        pass


def cpu_workers() -> int:
    """Host worker processes for the oracle: every core, bounded by memory
    (an agent step of this model holds about 0.6 GB)."""
    n = os.cpu_count() or 1
    try:
        import psutil

        n = min(n, max(1, int(psutil.virtual_memory().available / 0.75e9)))
    except Exception:  # noqa: BLE001
        pass
    return max(1, n)


class OraclePool:
    """Spawned process pool running oracle agent steps on all host cores."""

    def __init__(self, workers: int):
        import multiprocessing as mp

        self.workers = workers
        self.pool = mp.get_context("spawn").Pool(workers, initializer=_worker_init)

    def run(self, model, idx):
        A, B, C, D, obs = model
        tasks = [([a[b] for a in A], [x[b] for x in B], [c[b] for c in C], [d[b] for d in D], obs[b]) for b in idx]
        t0 = time.perf_counter()
        out = self.pool.map(_oracle_agent_step, tasks, chunksize=1)
        return out, time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def _max_rel(got, ref, floor):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    return float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), floor)))


def reduce_max_over_ranks(values, world: int, device="cpu") -> list:
    """Max over ranks of per-rank timings: the job takes as long as its slowest
    rank (every rank calls this, in the same order)."""
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


MINVAL = float(np.finfo(np.float64).eps)


class RefCpuStep:
    """The agent step on the reference's own CPU FFI kernels (``oracle/_ref``):
    the observed log-likelihood slices (``compute_log_likelihood_per_modality``,
    done here in NumPy as the reference does it in XLA before its FFI call),
    FpiCpu (16 iterations), NegEfeCpu over all 4096 policies (utility + state
    information gain, policy matrix broadcast over the batch as JAX's
    ``vmap_method="broadcast_all"`` passes it), q_pi = softmax(gamma G + log E)
    and the first-max action. The model is flattened once, outside the timed
    calls, as the GPU path does at ``Agent`` construction."""

    def __init__(self, model, idx):
        from oracle import efe as oefe
        from oracle import refcpu

        self.refcpu = refcpu
        A, B, C, D, obs = model
        idx = np.asarray(list(idx))
        n = len(idx)
        self.n = n
        flat = lambda xs: np.ascontiguousarray(np.concatenate(  # noqa: E731
            [np.asarray(x[idx], np.float32).reshape(n, -1) for x in xs], axis=1))
        self.A = [np.ascontiguousarray(a[idx]) for a in A]
        self.obs = obs[idx]
        self.A_flat, self.B_flat = flat(A), flat(B)
        self.C_flat = flat([np.repeat(c[:, None, :], T, 1) for c in C])
        self.lp = np.log(np.maximum(flat(D), MINVAL)).astype(np.float32)
        self.I = np.zeros((n, sum(S)), np.float32)
        self.pol = oefe.construct_policies(S, U, T).astype(np.int32)
        self.pm = np.ascontiguousarray(np.broadcast_to(self.pol, (n,) + self.pol.shape))
        F, M = len(S), len(O)
        self.A_deps, self.B_deps = [list(range(F))] * M, [[f] for f in range(F)]
        self.spans = refcpu.efe_spans(S, O, U, T, self.A_deps, self.B_deps)
        K = int(np.prod(S))
        self.ll_off = np.cumsum([0] + [K] * M)
        self.logE = np.log(np.full(len(self.pol), 1.0 / len(self.pol)))

    def __call__(self):
        n, K = self.n, int(np.prod(S))
        rows = np.arange(n)
        ll = np.concatenate([np.log(np.maximum(a[rows, self.obs[:, m]].reshape(n, K), MINVAL))
                             for m, a in enumerate(self.A)], axis=1).astype(np.float32)
        qs = self.refcpu.fpi_cpu(ll, self.lp, S, self.ll_off, self.A_deps, NUM_ITER)
        G = self.refcpu.neg_efe_cpu(self.pm, qs, self.A_flat, self.B_flat, self.C_flat, self.I, self.spans)
        z = GAMMA * G.astype(np.float64) + self.logE
        z -= z.max(axis=1, keepdims=True)
        q_pi = np.exp(z)
        q_pi /= q_pi.sum(axis=1, keepdims=True)
        return qs, G, q_pi, self.pol[np.argmax(q_pi, axis=1), 0]


def ref_cpu_available() -> bool:
    try:
        from oracle import ref_build

        ref_build.load()
        return True
    except Exception:  # noqa: BLE001
        return False


def ref_cpu_desc() -> str:
    from oracle import ref_build

    return (f"reference NegEfeCpu + FpiCpu (pymdp/ffi CPU kernels compiled from the reference's sources, "
            f"-O3 -ffast-math -march={ref_build.VARIANTS[ref_build.variant()]} -fopenmp, FP32), OpenMP on "
            f"{os.cpu_count()} host threads")


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the agent step on the same
    256-agent model, all of its agents every step (rank 0 only)."""
    if rank != 0:
        return
    n_agents = args.agents
    model = make_model(1234, n_agents)
    if not ref_cpu_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference's CPU FFI kernels) "
                          "was not built: run python -m oracle.ref_build where the reference sources are"}))
        return
    step = RefCpuStep(model, range(n_agents))
    for _ in range(max(1, args.warmup)):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = args.steps * n_agents / total
    line = {
        "impl": "reference", "metric": "agent-steps/s", "value": value, "unit": "agent-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload(n_agents), "agents_per_step": n_agents, "same_config": True},
        "cpu_baseline": {"value": value, "unit": "agent-steps/s", "cores": os.cpu_count(), "kind": "reference",
                         "sample": f"all {n_agents} agents of the workload per step: " + ref_cpu_desc()},
        "e2e": {"value": value, "unit": "agent-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def measure_peaks(dev) -> dict:
    """Dense-matmul peaks of this GPU measured in the run (best of 5 after
    warm-up, CUDA events): TF32 tensor cores (torch.matmul on FP32 with TF32
    allowed) and FP32 SIMT (the same matmul with TF32 disallowed). They are
    the roofline denominators of the TF32 and FP32-SIMT kernels; the HBM and
    BF16 figures come from MEASURED_PEAKS.json."""
    import torch

    n = 8192
    a = torch.randn((n, n), device=dev)
    b = torch.randn((n, n), device=dev)
    out = {}
    prev = torch.backends.cuda.matmul.allow_tf32
    try:
        for name, tf32 in (("tf32_tflops", True), ("fp32_simt_tflops", False)):
            torch.backends.cuda.matmul.allow_tf32 = tf32
            for _ in range(2):
                torch.matmul(a, b)
            best = float("inf")
            for _ in range(5):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                torch.matmul(a, b)
                e1.record()
                torch.cuda.synchronize(dev)
                best = min(best, e0.elapsed_time(e1))
            out[name] = 2.0 * n ** 3 / (best * 1e-3) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    out["how"] = f"torch.matmul FP32 {n}^3, TF32 allowed / disallowed, best of 5 (CUDA events)"
    return out


# Config 1: the plain single agent (S=[3,2], O=[3,5], U=[3,1], policy_len 1, 16 iterations, gamma 16).
C1_S, C1_O, C1_U = [3, 2], [3, 5], [3, 1]


def make_config1(seed: int):
    rng = np.random.default_rng(seed)

    def norm0(shape):
        x = rng.uniform(0, 1, size=shape)
        return (x / x.sum(0, keepdims=True)).astype(np.float32)

    A = [norm0((o, 3, 2)) for o in C1_O]
    B = [norm0((3, 3, 3)), norm0((2, 2, 1))]
    obs = rng.integers(0, np.array(C1_O), size=(1, len(C1_O))).astype(np.int32)
    return A, B, obs


def run_config1(dev, steps: int, warmup: int):
    """The plain single agent: one agent step (infer_states -> infer_policies
    -> sample_action) through ``Agent``, captured once in a CUDA graph and
    replayed; agent-steps/s = replays per second (launch/latency bound)."""
    import torch

    from pymdp_b200 import Agent

    A, B, obs = make_config1(5)
    agent = Agent(A, B, policy_len=1, gamma=16.0, batch_size=1, num_iter=NUM_ITER, device=dev)
    obs_d = torch.as_tensor(obs, device=dev)
    prior = [torch.full((1, s), 1.0 / s, device=dev) for s in C1_S]
    stream = torch.cuda.Stream(dev)

    def step():
        qs = agent.infer_states(obs_d, prior)
        q_pi, _ = agent.infer_policies(qs)
        return agent.sample_action(q_pi)

    with torch.cuda.stream(stream):
        for _ in range(max(warmup, 1)):
            step()
    torch.cuda.synchronize(dev)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        act = step()
    reps = 200
    for _ in range(max(warmup, 1)):
        graph.replay()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps * reps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize(dev)
    us = e0.elapsed_time(e1) * 1e3 / (steps * reps)
    # eager (no graph): the same calls launched one by one from Python
    t0 = time.perf_counter()
    for _ in range(steps * 20):
        step()
    torch.cuda.synchronize(dev)
    eager_us = (time.perf_counter() - t0) * 1e6 / (steps * 20)
    return {"workload": "plain single agent: S=[3,2], O=[3,5], U=[3,1], A/B uniform(0,1) normalised, C/D/E uniform, "
                        "policy_len 1, 16 FPI iterations, gamma 16; infer_states -> infer_policies -> sample_action",
            "agent_steps_per_s": 1e6 / us, "us_per_step_graph": us, "us_per_step_eager": eager_us,
            "action": act.cpu().tolist()}


def run_plain_config(dev, model, steps: int, warmup: int, flush):
    """The same agent step over the same 256 agents with the plain per-policy
    kernel: one thread per (agent, policy) in FP32 SIMT, every policy's full
    roll-out and contraction (no tensor cores, no shared policy prefixes). Its
    agent-steps/s is the denominator of the fused-vs-plain ratio."""
    import torch

    from pymdp_b200 import Agent

    A, B, C, D, obs = model
    agent = Agent(A, B, C=C, D=D, policy_len=T, gamma=GAMMA, batch_size=len(obs), num_iter=NUM_ITER, device=dev,
                  precision="fp32", efe_algorithm="dense")
    obs_d = torch.as_tensor(obs, device=dev)
    prior_d = [torch.as_tensor(d, device=dev) for d in D]

    def step():
        qs = agent.infer_states(obs_d, prior_d)
        q_pi, _ = agent.infer_policies(qs)
        return agent.sample_action(q_pi)

    for _ in range(max(1, warmup)):
        step()
    torch.cuda.synchronize(dev)
    evs = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        act = step()
        e1.record()
        evs.append((e0, e1))
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in evs) / steps
    return {"kernel": "efe_plain_kernel (FP32 SIMT, one thread per agent and policy) after the same fused FPI",
            "agent_steps_per_s": len(obs) / (ms * 1e-3), "ms_per_step": ms, "actions": act.cpu().numpy()}


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from pymdp_b200 import Agent, _lib

    sample = 0 if world > 1 else (cpu_workers() if args.cpu_sample is None else args.cpu_sample)
    n_agents = args.agents
    sample = min(sample, n_agents)
    pool = OraclePool(min(sample, cpu_workers())) if sample > 0 else None  # spawned before any GPU work
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    model = make_model(1234 + rank, n_agents)
    A, B, C, D, obs = model
    agent = Agent(A, B, C=C, D=D, policy_len=T, gamma=GAMMA, batch_size=n_agents, num_iter=NUM_ITER, device=dev,
                  precision=args.precision, efe_algorithm=args.efe)
    obs_d = torch.as_tensor(obs, device=dev)
    prior_d = [torch.as_tensor(d, device=dev) for d in D]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    main_only = args.legs == "main"
    fpi_res = None if main_only else run_fpi_config(dev, args.steps, args.warmup, flush)
    fpi_big = run_fpi_config(dev, args.steps, args.warmup, flush, 65536) if world == 1 and not main_only else None
    # single-GPU side measurements: run with N = 1 only
    extras = args.legs == "all" and world == 1
    peaks_run = measure_peaks(dev) if world == 1 and not main_only else {}
    fit_res = run_fit_config(dev, args.steps, args.warmup, flush) if extras else None
    ro_res = run_rollout_config(dev, min(args.steps, 5), args.warmup) if extras else None
    learn_res = run_learn_config(dev, args.steps, args.warmup, flush) if extras else None
    hmm_res = run_hmm_config(dev, args.steps, args.warmup, flush) if extras else None
    seq_res = run_seq_config(dev, args.steps, args.warmup, flush) if extras else None
    c1_res = run_config1(dev, args.steps, args.warmup) if world == 1 and not main_only else None
    plain_res = run_plain_config(dev, model, min(args.steps, 3), 1, flush) if world == 1 and not main_only else None

    def step():
        qs = agent.infer_states(obs_d, prior_d)
        q_pi, G = agent.infer_policies(qs)
        return agent.sample_action(q_pi)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        step()
    barrier()
    # outputs of one step, checked against the FP64 oracle on the CPU sample
    qs_chk = agent.infer_states(obs_d, prior_d)
    q_pi_chk, G_chk = agent.infer_policies(qs_chk)
    act_chk = agent.sample_action(q_pi_chk)
    chk = ([q[:, -1].cpu().numpy() for q in qs_chk], G_chk.cpu().numpy(), q_pi_chk.cpu().numpy(),
           act_chk.cpu().numpy())
    barrier()
    # eager steps (one Python call per kernel), for the record
    n0 = _lib.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    barrier()
    per_step_launches = (_lib.launch_count() - n0) // args.steps
    eager_ms = ev0.elapsed_time(ev1) / args.steps
    # the timed step: the whole agent step captured as one CUDA graph and replayed, inputs resident (its launches
    # chained by programmatic dependent launch throughout). The same step as two graphs (belief update | policies
    # + action), replayed after the timed steps with an event between them, times the neg-EFE launch for the
    # roofline.
    gfull = agent.capture_step(warmup=args.warmup)
    gstep = agent.capture_step(warmup=args.warmup, split=True)
    flat_prior = torch.cat([p.reshape(n_agents, -1) for p in prior_d], dim=1)
    for g in (gfull, gstep):
        g.obs.copy_(obs_d)
        g.prior.copy_(flat_prior)
    (g_full,) = gfull.graphs
    g_states, g_policies = gstep.graphs
    for _ in range(args.warmup):
        gfull.step()
        gstep.step()
    barrier()
    graph_same = int((gfull.action.cpu().numpy() == chk[3]).all(axis=1).sum())
    split_same = int((gstep.action.cpu().numpy() == chk[3]).all(axis=1).sum())
    evs, efe_ev = [], []
    with ClockSampler(local_rank) as clocks:
        # nvidia-smi answers every 0.2 s or so, far longer than the timed steps take: identical untimed
        # steps (flush + the step's graph) run until the sampler holds three readings under this load (2 s at
        # most), and the timed steps follow with no gap
        t_end = time.time() + 2.0
        while len(clocks.rows) < 3 and time.time() < t_end:
            for _ in range(20):
                flush.zero_()
                g_full.replay()
            torch.cuda.synchronize()
        barrier()
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
            e0.record(stream)
            g_full.replay()
            e1.record(stream)
            evs.append((e0, e1))
        barrier()
        # the neg-EFE launch alone, for the roofline: same flush, belief update untimed
        for _ in range(args.steps):
            flush.zero_()
            g_states.replay()
            em, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
            em.record(stream)
            g_policies.replay()
            e1.record(stream)
            efe_ev.append((em, e1))
        barrier()
    launches = args.steps * per_step_launches
    ms = sum(a.elapsed_time(b) for a, b in evs)
    efe_ms = sum(a.elapsed_time(b) for a, b in efe_ev) / len(efe_ev)
    # e2e through the public API (Agent.capture_pipeline -> PipelinedAgentStep.step) with host buffers: every
    # step copies pinned observations and prior in and its action out, on copy streams beside the compute of
    # the neighbouring steps; the timed region starts before the first input copy and ends after the last
    # action has landed in host memory
    pipe = agent.capture_pipeline(warmup=1)
    obs_h = torch.as_tensor(obs).pin_memory()
    prior_h = torch.cat([torch.as_tensor(d).reshape(n_agents, -1) for d in D], dim=1).pin_memory()
    act_h = torch.empty((n_agents, len(S)), dtype=torch.int32).pin_memory()

    def e2e_step():
        pipe.step(obs_h, prior_h, act_h)

    for _ in range(args.warmup):
        e2e_step()
    pipe.drain()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    pipe.begin(ev0)
    for _ in range(args.steps):
        e2e_step()
    pipe.drain()
    ev1.record(stream)
    barrier()
    e2e_ms = ev0.elapsed_time(ev1)
    e2e_same = int((act_h.numpy() == chk[3]).all(axis=1).sum())
    h2d = obs_h.numel() * 4 + prior_h.numel() * 4
    d2h = act_h.numel() * 4
    ms, e2e_ms, efe_ms = reduce_max_over_ranks([ms, e2e_ms, efe_ms], world, dev)
    if rank != 0:
        if pool is not None:
            pool.close()
        return
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:  # noqa: BLE001
        pass
    factored = args.efe == "factored"
    tree = agent.precision != "fp32"  # the tensor-core paths evaluate each policy prefix once
    if agent.precision == "tf32x3" and "tf32_tflops" in peaks_run:
        peak_tf, peak_src = peaks_run["tf32_tflops"], "TF32 dense matmul measured in this run (torch.matmul, TF32)"
    elif agent.precision == "fp32" and "fp32_simt_tflops" in peaks_run:
        peak_tf, peak_src = peaks_run["fp32_simt_tflops"], "FP32 SIMT matmul measured in this run"
    else:
        peak_tf = peaks.get("bf16_tflops", 1590.0)
        peak_src = "MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else "fallback"
    peak_gbs = peaks.get("hbm_gbs", 6650.0)
    flops = efe_flops_per_agent(tree) * n_agents
    dense_flops = efe_flops_per_agent(False) * n_agents
    achieved_tf = flops / (efe_ms * 1e-3) / 1e12
    total_agents = n_agents * world
    value = total_agents * args.steps / (ms * 1e-3)
    err = None
    if pool is not None:
        try:
            ref, _ = pool.run(model, range(sample))
        finally:
            pool.close()
        qs_g, G_g, q_pi_g, act_g = chk
        err = {
            "agents": sample,
            "qs_max_rel": max(_max_rel(qs_g[f][b], ref[b][0][f], 1e-6) for b in range(sample) for f in range(len(S))),
            "G_max_rel": max(_max_rel(G_g[b], ref[b][1], 1e-6) for b in range(sample)),
            "G_max_abs_over_max_G": max(float(np.max(np.abs(np.asarray(G_g[b], np.float64) - ref[b][1]))
                                            / np.max(np.abs(ref[b][1]))) for b in range(sample)),
            "q_pi_max_abs": max(float(np.max(np.abs(q_pi_g[b] - ref[b][2]))) for b in range(sample)),
            "actions_equal": int(sum(bool(np.array_equal(act_g[b], ref[b][3])) for b in range(sample))),
        }
    cpu_base = None
    if world == 1 and ref_cpu_available() and args.cpu_sample != 0:
        # the reference's own CPU agent step on a bounded sample of the same agents (about 10-30 s of CPU work)
        n_ref = min(n_agents, args.ref_sample)
        rstep = RefCpuStep(model, range(n_ref))
        rstep()
        reps, t0 = 0, time.perf_counter()
        while reps < 2 or (time.perf_counter() - t0 < 10.0 and reps < 20):
            rstep()
            reps += 1
        dt = time.perf_counter() - t0
        cpu_base = {"value": reps * n_ref / dt, "unit": "agent-steps/s", "cores": os.cpu_count(), "kind": "reference",
                    "sample": f"agents 0..{n_ref - 1} of the timed model x {reps} steps ({dt:.1f} s): "
                              + ref_cpu_desc()}
    fused_over_plain = None
    if plain_res is not None:
        fused_over_plain = value / plain_res["agent_steps_per_s"]
        plain_res["actions_equal_fused"] = int((plain_res.pop("actions") == chk[3]).all(axis=1).sum())
    line = {
        "metric": "agent-steps/s", "value": value, "unit": "agent-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload(n_agents), "agents_per_gpu": n_agents, "fpi_iters": NUM_ITER, "policies": 4096,
                   "efe_algorithm": args.efe, "precision": "fp32 (factored)" if factored else agent.precision, "l2": "flushed (256 MiB write) between timed steps",
                   "parallelism": f"agents sharded over {world} GPU(s), no collective"},
        "e2e": {"value": total_agents * args.steps / (e2e_ms * 1e-3), "unit": "agent-steps/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "form": "Agent.capture_pipeline: each step's copies on copy streams beside the neighbouring steps' "
                        "compute (two buffer sets); the region ends after the last action reached host memory",
                "l2": "not flushed between steps: the model's A (218 MB at 256 agents) exceeds the 126 MB L2"},
        "gpu_launches": int(launches),
        "step_form": {"timed": "CUDA graph replay (the whole step as one graph; the neg-EFE launch timed on the "
                               "two-graph form, belief update | policies + action)",
                      "kernels_per_step": per_step_launches, "eager_ms_per_step": eager_ms,
                      "graph_actions_equal_eager": graph_same, "split_graph_actions_equal_eager": split_same,
                      "e2e_actions_equal_eager": e2e_same},
        "fused_over_plain": fused_over_plain,
        "plain": plain_res,
        "config1": c1_res,
        "roofline": ({"bound": "hbm", "achieved": efe_bytes_per_agent() * n_agents / (efe_ms * 1e-3) / 1e9,
                      "peak": peak_gbs, "unit": "GB/s",
                      "frac": efe_bytes_per_agent() * n_agents / (efe_ms * 1e-3) / 1e9 / peak_gbs,
                      "traffic": (EFE_TRAFFIC_PER_AGENT["factored"] * n_agents
                                  if "factored" in EFE_TRAFFIC_PER_AGENT else None),
                      "kernel": f"factored neg-EFE launch over {n_agents} agents (history marginals, level 1, "
                                f"tail, combine) + q_pi",
                      "bytes_per_launch": efe_bytes_per_agent() * n_agents, "ms_per_launch": efe_ms,
                      "executed_flops_per_launch": efe_factored_flops_per_agent() * n_agents,
                      # the same launch against the FP32 SIMT peak measured in this run: the tail's
                      # contractions and entropies make it compute-bound as much as HBM-bound
                      "executed_tflops": efe_factored_flops_per_agent() * n_agents / (efe_ms * 1e-3) / 1e12,
                      "fp32_simt_peak_tflops": peaks_run.get("fp32_simt_tflops"),
                      "fp32_simt_frac": (efe_factored_flops_per_agent() * n_agents / (efe_ms * 1e-3) / 1e12
                                         / peaks_run["fp32_simt_tflops"]) if "fp32_simt_tflops" in peaks_run else None,
                      "dense_equivalent_flops_per_launch": dense_flops,
                      "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback"}
                     if factored else
                     {"bound": "tensor", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
                      "frac": achieved_tf / peak_tf,
                      "traffic": (EFE_TRAFFIC_PER_AGENT[agent.precision] * n_agents
                                  if agent.precision in EFE_TRAFFIC_PER_AGENT else None),
                      "kernel": f"neg-EFE launch over {n_agents} agents (policy evaluation + q_pi)",
                      "flops_per_launch": flops, "ms_per_launch": efe_ms,
                      "policy_tree": tree, "dense_equivalent_flops_per_launch": dense_flops,
                      "dense_equivalent_tflops": dense_flops / (efe_ms * 1e-3) / 1e12,
                      "dense_equivalent_frac": dense_flops / (efe_ms * 1e-3) / 1e12 / peak_tf,
                      "peak_source": peak_src}),
        "peaks_measured": peaks_run or None,
        "cpu_baseline": cpu_base,
        "error_vs_fp64": err,
        "fpi": None if fpi_res is None else dict(
            fpi_res, roofline={"bound": "hbm", "achieved": fpi_res["gbs"], "peak": peak_gbs, "unit": "GB/s",
                               "frac": fpi_res["gbs"] / peak_gbs}),
        "fpi_65536": None if fpi_big is None else dict(
            fpi_big, roofline={"bound": "hbm", "achieved": fpi_big["gbs"], "peak": peak_gbs, "unit": "GB/s",
                               "frac": fpi_big["gbs"] / peak_gbs}),
        "fit": fit_res,
        "rollout": ro_res,
        "learn": learn_res,
        "hmm": hmm_res,
        "seq": seq_res,
        "clocks": dict(clocks.summary(), window="identical untimed steps run just before the timed steps, "
                                               "then the timed steps"),
    }
    print(json.dumps(line), flush=True)


def relaunch_under_torchrun(n: int):
    """``--gpus N`` without a torchrun environment: run this same command as N
    ranks (one process per GPU) under torch.distributed.run on 127.0.0.1."""
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *sys.argv[1:]]
    raise SystemExit(subprocess.call(cmd))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="step", choices=["step", "fpi", "fit", "rollout", "learn", "hmm", "seq"],
                    help="step: the agent step (default); fpi: only the 4096-agent FPI model; fit: only the "
                         "model-fitting gradient; rollout: only the uneven-size rollout (for profiling)")
    ap.add_argument("--legs", default="all", choices=["all", "step", "main"],
                    help="all: also the fitting, rollout, learning and HMM workloads (default); step: the agent step "
                         "with its FPI, config-1, plain-kernel and peak legs; main: the agent step alone (profiling)")
    ap.add_argument("--hmm-agents", type=int, default=HMM_AGENTS, help="agents of the hmm workload")
    ap.add_argument("--fpi-agents", type=int, default=FPI_AGENTS, help="agents of the fpi workload")
    ap.add_argument("--agents", type=int, default=AGENTS, help="agents per GPU (256 = the benchmark workload)")
    ap.add_argument("--cpu-sample", type=int, default=None, help="agents in the FP64 check sample (0 = skip)")
    ap.add_argument("--ref-sample", type=int, default=64,
                    help="agents per step of the reference CPU baseline sample (b200 arm)")
    ap.add_argument("--efe", default="factored", choices=["factored", "dense"],
                    help="neg-EFE algorithm: factored (contraction factor by factor over the per-factor marginals "
                         "of the policy tree) or dense (one contraction per policy prefix, at --precision)")
    ap.add_argument("--precision", default="tf32x3", choices=["fp32", "tf32x3", "bf16"],
                    help="dense EFE contraction: fp32 (SIMT), tf32x3 or bf16 (tcgen05 tensor cores)")
    args = ap.parse_args()
    if args.gpus < 1:
        raise SystemExit("--gpus must be >= 1")
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        relaunch_under_torchrun(args.gpus)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}: launch one rank per GPU")
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload != "step" and world > 1:
        raise SystemExit("--workload fpi/fit/rollout/learn/hmm runs on one GPU")
    if args.workload != "step":
        import torch

        dev = torch.device("cuda", local_rank)
        torch.cuda.set_device(dev)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        if args.workload == "fpi":
            res = run_fpi_config(dev, args.steps, args.warmup, flush, args.fpi_agents)
        elif args.workload == "fit":
            res = run_fit_config(dev, args.steps, args.warmup, flush)
        elif args.workload == "rollout":
            res = run_rollout_config(dev, args.steps, args.warmup)
        elif args.workload == "hmm":
            res = run_hmm_config(dev, args.steps, args.warmup, flush, args.hmm_agents)
        elif args.workload == "seq":
            res = run_seq_config(dev, args.steps, args.warmup, flush)
        else:
            res = run_learn_config(dev, args.steps, args.warmup, flush)
        print(json.dumps(res), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
