"""The multi-GPU (replica) path's host logic on CPU: two ranks over gloo take the max of
their times the way bench.py's ranks do over NCCL, and bench.py's reference arm runs under
torchrun with two ranks (rank 0 measures and prints, the other exits without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from hindemith_b200.replicas import job_rate, max_over_ranks, rank_seed

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        times = max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * (rank + 1)])
        res = {"times": times, "seed": rank_seed(1000, rank),
               "rate": job_rate(100.0, world, times[0])}
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["times"] == [2.0, 10.0, 1.0]  # the slowest rank's time, on every rank
        assert r["rate"] == 100.0 * world / 2.0
    assert [r["seed"] for r in res] == [1000, 1001]


def test_max_over_ranks_without_a_group():
    from hindemith_b200.replicas import max_over_ranks

    assert max_over_ranks([3, 1.5]) == [3.0, 1.5]


def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "3", "--cpu-sample-sweeps", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
