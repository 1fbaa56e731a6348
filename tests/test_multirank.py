"""World-size-2 checks of the replica plumbing bench.py uses on N GPUs, run
as two gloo ranks on the CPU: every rank takes the same collective steps,
throughput is all ranks' units over the slowest rank's time, and the CPU
reference arm runs on rank 0 only."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    units = 1000.0 * (rank + 1)      # rank 1 adapted twice the tets
    ms = 10.0 + 30.0 * rank          # and was slower
    value, ms_max, total = bench.replica_throughput(units, ms, world)
    bench.barrier(world)
    ref = bench.run_reference if rank else None
    out[rank] = (value, ms_max, total, ref is not None)
    dist.destroy_process_group()


def test_replica_throughput_two_ranks():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        value, ms_max, total, _ = out[r]
        assert ms_max == 40.0
        assert total == 3000.0
        assert abs(value - 3000.0 / 0.040) < 1e-6


def _ref_worker(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import argparse
    import bench
    args = argparse.Namespace(steps=1, warmup=0)
    if rank != 0:
        out[rank] = bench.run_reference(args, world, rank)
    else:
        out[rank] = "rank0-would-run"
    dist.barrier()
    dist.destroy_process_group()


def test_reference_arm_runs_on_rank0_only():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_ref_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[1] is None
