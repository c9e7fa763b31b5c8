"""The N > 1 host path of bench.py on CPU: two ranks on the gloo backend over
127.0.0.1. Agents are independent, so ranks share nothing but the timing
reduction: the job's time is the slowest rank's (max over ranks), the
reference arm runs on rank 0 only, and each rank builds its own agents."""

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import io
    import contextlib

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        red = bench.reduce_max_over_ranks([1.0 + rank, 10.0 - rank, 3.5], world)
        args = type("A", (), dict(agents=8, steps=1, warmup=1, gpus=world))()
        buf = io.StringIO()
        if rank != 0:
            with contextlib.redirect_stdout(buf):
                bench.run_reference(args, rank, world)  # other ranks exit without work
        A0 = bench.make_model(1234 + rank, 2)[0][0]
        dist.barrier()
        out.put((rank, red, buf.getvalue(), float(np.asarray(A0).sum()), float(np.asarray(A0).ravel()[0])))
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_timing_rank0_reference_and_distinct_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, red0, out0, s0, a0), (r1, red1, out1, s1, a1) = res
    assert red0 == red1 == [2.0, 10.0, 3.5]
    assert out1 == ""
    assert a0 != a1  # each rank draws its own agents (seed 1234 + rank)


@pytest.mark.parametrize("world", [1])
def test_reduce_is_identity_on_one_rank(world):
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max_over_ranks([3.0, 1.5], world) == [3.0, 1.5]


def _run_bench(args, env_extra=None, timeout=240):
    import json
    import subprocess

    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                              "MASTER_PORT")}
    env.update(env_extra or {})
    res = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                         env=env, timeout=timeout, cwd=ROOT)
    lines = [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]
    return res, lines


def test_gpus_flag_launches_one_rank_per_gpu_for_the_reference_arm():
    """``bench.py --gpus 2`` outside torchrun relaunches itself as 2 ranks
    (torch.distributed.run on 127.0.0.1); the reference arm runs on rank 0
    alone and prints one line whose n_gpus is the world size."""
    from oracle import ref_build
    if not ref_build.build():
        pytest.skip("reference CPU kernels not built")
    res, lines = _run_bench(["--impl", "reference", "--gpus", "2", "--agents", "4", "--steps", "1",
                             "--warmup", "1"])
    assert res.returncode == 0, res.stderr[-2000:]
    assert len(lines) == 1, res.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["config"]["same_config"]


def test_gpus_flag_must_match_the_launched_world():
    res, lines = _run_bench(["--impl", "reference", "--gpus", "2", "--agents", "4"],
                            env_extra={"WORLD_SIZE": "1", "RANK": "0", "LOCAL_RANK": "0"})
    assert res.returncode != 0 and not lines
    assert "launch one rank per GPU" in res.stderr
