"""The multi-rank path on CPU (gloo, world size 2): the benchmark runs one
replica per rank with no data-path collective and reports the max over ranks;
the reference arm prints one line from rank 0 and lets the others exit."""
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


def _max_worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sys.path.insert(0, ROOT)
        import bench

        out[rank] = bench.max_over_ranks(dist, 1.5 + rank)  # each rank's own time
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp

    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_max_worker, args=(2, port, out), nprocs=2, join=True)
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_reference_arm_two_ranks():
    """torchrun with 2 CPU ranks: one JSON line (rank 0), exit status 0."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--latt", "4", "4", "4", "8"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["cpu_baseline"]["kind"] == "port" and rec["e2e"]["h2d_bytes_per_step"] == 0


@pytest.mark.parametrize("world", [2])
def test_replica_seeds_differ(world):
    """Replicas solve independent systems: each rank seeds its own gauge field
    and source (bench.py: seed + rank)."""
    sys.path.insert(0, ROOT)
    import bench

    seeds = {(bench.GAUGE_SEED + r, bench.SRC_SEED + r) for r in range(world)}
    assert len(seeds) == world
