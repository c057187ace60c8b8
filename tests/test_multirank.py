"""CPU tests of the multi-rank (replica) path of bench.py with the gloo
backend, world size 2: the max-over-ranks timing, the whole-job throughput of
independent replicas, and that the reference arm under torchrun prints one
line from rank 0 only."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t_ms = 100.0 + 50.0 * rank  # rank 1 is the slowest
    t_max = bench.max_over_ranks(t_ms, dist, "cpu")
    value = bench.replica_throughput(1000, 4, t_max, world)
    dist.barrier()
    dist.destroy_process_group()
    Path(out_dir, f"rank{rank}.json").write_text(json.dumps({"t_max": t_max, "value": value}))


def test_max_over_ranks_and_replica_throughput_gloo(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        d = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert d["t_max"] == 150.0
        assert d["value"] == pytest.approx(2 * 1000 * 4 / 0.150)


def test_reference_arm_under_torchrun_prints_rank0_only():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"), "--gpus", "2",
           "--impl", "reference", "--workload", "c1", "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=str(ROOT), env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
