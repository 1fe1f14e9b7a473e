"""The benchmark's multi-process path on CPU (gloo, world size 2).

Lattices are independent, so N ranks run N replicas of the workload with no
data-path collective; the only cross-rank steps are the barriers around the
timed region and the max-over-ranks reduction of the device time.  These
tests run that plumbing with two gloo ranks on the host: the reduction gives
every rank the slowest rank's time, and `bench.py --impl reference` under
torchrun prints exactly one JSON line (rank 0) while the other rank exits 0
without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist, r, w, local = bench.dist_init(world)
    assert (r, w, local) == (rank, world, rank)
    bench.barrier(dist)
    slowest = bench.max_over_ranks(dist, 10.0 + 5.0 * rank)  # per-rank device ms
    bench.barrier(dist)
    with open(f"{out_path}.{rank}", "w") as f:
        f.write(repr(slowest))
    dist.destroy_process_group()


def test_max_over_ranks_gives_every_rank_the_slowest_time(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    out = str(tmp_path / "slowest")
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        with open(f"{out}.{r}") as f:
            assert float(f.read()) == 15.0


def test_reference_arm_under_torchrun_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--cpu-L", "64"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["unit"] == d["e2e"]["unit"] == "spin-flip attempts/ns"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
