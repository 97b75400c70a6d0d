"""The N > 1 path of bench.py on CPU (gloo, world size 2).

Blocks are independent, so several GPUs run replicas of the benchmark step
with no collective on the data path; the ranks only meet at barriers and in
the max-over-ranks of the step time.  Those pieces, and the reference arm's
rank-0-only rule, are checked here with CPU processes.
"""

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    import bench

    dist.barrier()
    got = bench.max_over_ranks(dist, 1.5 + rank, "cpu")
    dist.barrier()
    Path(out_dir, f"rank{rank}.txt").write_text(repr(got))
    dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    mp.start_processes(_rank_main, args=(free_port(), str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    assert [float((tmp_path / f"rank{r}.txt").read_text()) for r in range(2)] == [2.5, 2.5]


def test_reference_arm_prints_one_line_from_rank_zero():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={free_port()}", str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--size", "32"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
    # The same workload config as the GPU arm's line (how the arm samples it
    # is stated beside it).
    import bench

    assert d["config"] == bench.workload_config(32, 2) and "slab" in d["sample"]
