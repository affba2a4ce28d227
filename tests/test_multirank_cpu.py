"""World-size-2 gloo check of bench.py's multi-rank bookkeeping (replicas, max over ranks)."""
import os
import socket
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, device="cpu")
    value = bench.aggregate_rate(world, steps=4, cells=1000, ms=ms)
    out[rank] = (ms, value)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_max_and_aggregate():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn")
    assert out[0][0] == out[1][0] == 15.0
    assert abs(out[0][1] - 2 * 4 * 1000 / 0.015) < 1e-6
