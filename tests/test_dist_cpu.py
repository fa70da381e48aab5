"""The multi-rank logic of bench.py on the CPU: two gloo ranks.  Each rank
solves its own independent batch (no exchange on the data path); the job's
throughput is the eigenpairs of all ranks over the slowest rank's time."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from mr3smp_b200 import workloads as wl


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        b = bench.rank_batch(wl, 16, 3, 256, rank)
        ns = [len(D) for D, E, _ in b]
        ms = [120.0, 300.0][rank]              # rank 1 is the slow one
        value, ms_per_step = bench.job_throughput(dist, "cpu", ms, 3, sum(ns))
        out[rank] = (ns, value, ms_per_step)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ws, port = 2, _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(ws, port, out), nprocs=ws, join=True, start_method="spawn")
    ns0, v0, t0 = out[0]
    ns1, v1, t1 = out[1]
    assert ns0 != ns1                           # independent batches per rank
    assert t0 == t1 == pytest.approx(100.0)     # slowest rank: 300 ms over 3 steps
    assert v0 == v1 == pytest.approx((sum(ns0) + sum(ns1)) / 0.1)
