"""World-size-2 checks of the multi-GPU plumbing bench.py uses on N GPUs,
run as two gloo ranks on the CPU: every rank takes the same collective
steps, throughput is all ranks' units over the slowest rank's time, the CPU
reference arm runs on rank 0 only, and meshes placed whole on the ranks by
bin packing (each rank adapting its own with the oracle) end as they do on
one rank."""
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


def _adapt_worker(rank, world, port, out):
    """Each rank adapts the meshes placed on it (the oracle on the CPU
    stands in for a GPU) and reports their digests; the ranks exchange only
    the final counts, as bench.py's batched legs do."""
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    import bench
    import large_flows as F
    from oracle import oracle as O
    from omega_h_v1_b200 import workloads as W
    jobs = W.batched_boxes(12, seed=5, nmax=5)
    mine = W.place_jobs(jobs, world)[rank]
    digests, tets = {}, 0.0
    for i in mine:
        m = F.box_job_mesh(O.Oracle, O.box, jobs[i])
        m.adapt(*F.BOX_ADAPT)
        digests[i] = O.snapshot_digest(m.snapshot())
        tets += m.count(3)
        m.close()
    total = bench.sum_over_ranks(tets, world)
    out[rank] = (mine, digests, total)
    dist.destroy_process_group()


def test_meshes_placed_on_two_ranks_adapt_as_on_one():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import large_flows as F
    from oracle import oracle as O
    from omega_h_v1_b200 import workloads as W
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_adapt_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    jobs = W.batched_boxes(12, seed=5, nmax=5)
    placed = sorted(out[0][0] + out[1][0])
    assert placed == list(range(len(jobs)))           # every mesh placed once
    want, tets = {}, 0
    for i, j in enumerate(jobs):
        m = F.box_job_mesh(O.Oracle, O.box, j)
        m.adapt(*F.BOX_ADAPT)
        want[i] = O.snapshot_digest(m.snapshot())
        tets += m.count(3)
        m.close()
    for r in range(world):
        for i, d in out[r][1].items():
            assert d == want[i], (r, i)
        assert out[r][2] == tets


def test_placement_balances_estimated_work():
    from omega_h_v1_b200 import workloads as W
    jobs = W.batched_boxes()
    for nb in (1, 2, 4, 8):
        bins = W.place_jobs(jobs, nb)
        assert sorted(i for b in bins for i in b) == list(range(len(jobs)))
        loads = [sum(jobs[i].estimated_output_tets() for i in b) for b in bins]
        biggest = max(j.estimated_output_tets() for j in jobs)
        # greedy largest-first: no bin exceeds the mean by more than one job
        assert max(loads) <= sum(loads) / nb + biggest
