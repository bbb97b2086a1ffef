"""The multi-rank logic of bench.py on CPU: two gloo ranks on 127.0.0.1.

bench.py --gpus N runs N independent replicas of the timestep (one per GPU; a timestep has
no partition that needs a collective), so the only cross-rank steps are the barriers and
the reduction of each timed interval to its maximum over ranks.  Here:
* max_over_ranks gives every rank the largest of the ranks' values (device and end-to-end
  times alike), and the bare value without a process group;
* the whole-job throughput built from it, world x steps / max time, counts every rank's
  steps at the slowest rank's pace;
* the reference arm (--impl reference) does its work on rank 0 only: another rank returns
  at once and prints nothing.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(dist, 10.0 + 5.0 * rank, "cpu")    # rank 1 is the slower one
        e2e = bench.max_over_ranks(dist, 0.004 if rank == 0 else 0.003, "cpu")
        dist.barrier()
        out.put((rank, ms, e2e))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == 15.0 and g[2] == 0.004 for g in got), got
    # whole-job throughput as bench.py forms it: world x steps / max time
    steps, world = 20, 2
    assert world * steps / (got[0][1] * 1e-3) == 2 * 20 / 0.015


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 3.25, "cpu") == 3.25


def test_reference_arm_other_ranks_do_nothing():
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    args = argparse.Namespace(workload="dynamo128", steps=3, warmup=3, slices=5)
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args, 1, 2)
    assert buf.getvalue() == ""
