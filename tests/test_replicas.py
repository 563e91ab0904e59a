"""The multi-process side of bench.py on the CPU: world_size-2 gloo ranks
take the job's time as the slowest rank's and the rate over all ranks' units;
the reference arm runs on rank 0 alone.  No GPU."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(REPO))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
        rate = bench.job_rate(1000, ms, world)
        rows = bench.sum_over_ranks(100 + rank, world, "cpu")
        q.put((rank, ms, rate, rows))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[1] for g in got] == [15.0, 15.0]
    assert all(abs(g[2] - 2 * 1000 / 0.015) < 1e-6 for g in got)
    assert [g[3] for g in got] == [201.0, 201.0]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(REPO))
    import bench
    assert bench.max_over_ranks(7.5, 1, "cpu") == 7.5
    assert bench.job_rate(500, 250.0, 1) == 2000.0


@pytest.mark.parametrize("rank", [0, 1])
def test_reference_arm_runs_on_rank_zero_only(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload",
                          "small", "--steps", "1", "--warmup", "0", "--gpus", "2"],
                         cwd=REPO, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    if rank:
        assert lines == []
    else:
        d = json.loads(lines[-1])
        assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
        assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
