"""The multi-GPU plumbing of bench.py on CPU ranks (gloo, world size 2):
each rank times its own replica, the job takes the slowest rank's time, and
only rank 0 reports; the reference arm under two ranks prints one line."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    ranks = bench.Ranks(dist, "cpu")
    ranks.barrier()
    ms_local = 100.0 + 50.0 * rank  # rank 1 is the slow one
    ms = ranks.allmax(ms_local)
    value = bench.replica_throughput(1000, 10, world, ms)
    ranks.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, value))


def test_allmax_and_throughput_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value in out:
        assert ms == 150.0  # the slowest rank's time on every rank
        assert value == pytest.approx(1000 * 10 * 2 / 0.150)


def test_reference_arm_under_two_ranks_prints_one_line():
    port = 29700 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--workload", "shell16"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0


def test_path_bytes_follow_the_compulsory_state_traffic():
    """Algorithmic bytes per zone-update of the path: every stage reads and
    writes the 12-word state (60 B in the precision form), later stages also
    read the stage-start copy: RK2 / IMEX-RK2 480 B (300 B), SSP-RK3 768 B
    (480 B)."""
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.path_bytes_per_zone_update(2, False) == 480.0
    assert bench.path_bytes_per_zone_update(4, False) == 480.0
    assert bench.path_bytes_per_zone_update(4, True) == 300.0
    assert bench.path_bytes_per_zone_update(3, False) == 768.0
    assert bench.path_bytes_per_zone_update(3, True) == 480.0
