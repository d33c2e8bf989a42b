"""Multi-GPU form of the benchmark is replicas only: each rank renders its own
frames, and the job time is the slowest rank's (max over ranks).  This checks
the host-side aggregation with two gloo ranks on the CPU."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local_ms = [100.0, 250.0][rank]
    res = bench.aggregate(local_ms, steps=10, world=world, pixels=2_073_600,
                          triangles=1_470_464, dist=dist, device="cpu")
    q.put((rank, res))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_aggregation():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0] == out[1]
    total, mpix, mtri = out[0]
    assert total == 250.0
    assert mpix == pytest.approx(2 * 10 * 2_073_600 / (250.0 * 1e3))
    assert mtri == pytest.approx(2 * 10 * 1_470_464 / (250.0 * 1e3))
