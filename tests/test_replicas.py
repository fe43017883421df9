"""Multi-process (N > 1) plumbing of bench.py on CPU with gloo, world size 2: the path runs as
independent replicas (no data-path collective), so what the ranks share is the timing
reduction (max over ranks), the barriers around the timed region, and rank-0-only output."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(world)
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow replica
        out[rank] = bench.reduce_max(ms, world)
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_gloo():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert dict(out) == {0: 15.0, 1: 15.0}


@pytest.mark.parametrize("rank", [0, 1])
def test_reference_arm_prints_on_rank_zero_only(rank):
    env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "rbc2d",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if rank == 0:
        assert len(lines) == 1
        d = json.loads(lines[0])
        assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
        assert d["e2e"]["value"] == d["value"]
        # the warm-up steps run untimed; the timed count and the requested count are reported
        assert d["warmup"] == 3 and d["steps"] == 1 and d["steps_requested"] == 1
        for k in ("metric", "unit", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "dtype", "config"):
            assert k in d, k
    else:
        assert lines == []
