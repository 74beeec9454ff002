"""The benchmark's multi-rank host logic on CPU: two ranks over gloo (127.0.0.1),
the way `python -m torch.distributed.run --nproc-per-node 2 bench.py` runs them
on GPUs (where the backend is NCCL).  Checks that the step time is the maximum
over the ranks on every rank, that the whole-job value counts every rank's
systems, that every replica solves its own systems, and that the reference arm
does its work on rank 0 alone."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 5.0 + 2.0 * rank  # rank 1 is the slower replica
        t = bench.reduce_max_ms(ms, world, dist, "cpu")
        v = bench.aggregate_value(world, 1000, t)
        dist.barrier()
        # the reference arm: rank 0 alone works; the others return at once
        class A:
            pass
        args = A()
        ref_rc = bench.run_reference(args) if rank != 0 else None
        out.put((rank, t, v, bench.rank_seed(rank), ref_rc))
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_time_and_whole_job_value():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(2))
    (r0, t0, v0, s0, _), (r1, t1, v1, s1, rc1) = res
    assert (r0, r1) == (0, 1)
    assert t0 == t1 == 7.0                      # max over the ranks, the same on both
    assert v0 == v1 == pytest.approx(2 * 1000 / 7.0e-3)
    assert s0 != s1 and s0 == 1000               # own systems per replica; rank 0's are the reference arm's
    assert rc1 == 0                              # the reference arm's non-zero ranks do no work
