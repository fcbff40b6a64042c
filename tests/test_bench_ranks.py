"""The multi-process (N > 1) paths of bench.py on the CPU: the max-over-ranks
job time with two gloo ranks, and the reference arm under torchrun, where
rank 0 alone measures and prints."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    # each rank's own step time; the job is as slow as the slowest rank
    ms = [12.5, 40.0][rank]
    job_ms = bench.max_over_ranks(ms, dist, "cpu")
    out[rank] = (job_ms, bench.whole_job_rate(1000, 10, world, job_ms * 1e-3))
    dist.barrier()
    dist.destroy_process_group()


def test_job_time_is_the_slowest_rank():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1]
    job_ms, rate = res[0]
    assert job_ms == 40.0
    # 2 replicas x 1000 updates x 10 steps in 40 ms
    assert rate == pytest.approx(2 * 1000 * 10 / 0.040 / 1e6)


def test_reference_arm_under_torchrun_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "3", "--workload", "tgv64",
           "--ref-seconds", "2"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
