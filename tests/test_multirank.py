"""Multi-rank plumbing of bench.py on CPU: two gloo ranks.

Under torchrun every rank runs its own replica of the workload on its own GPU
(the transforms are independent, so there is no data-path collective); the
only cross-rank steps are barriers and the reduction of each timed region to
the slowest rank.  These tests run bench.py's own helpers for those steps in
two processes joined by a gloo process group on 127.0.0.1 (world size 2), the
way the NCCL group joins them on GPUs: both ranks must see the slowest rank's
time, the reported throughput must count both replicas' work over that time,
and the reference arm must run on rank 0 only.
"""
import contextlib
import datetime
import io
import os
import socket
import sys
import types

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # the device-timed region (ms) and the end-to-end region (s) differ per rank
        ms = bench.max_over_ranks(dist, 10.0 * (rank + 1), "cpu")
        el = bench.max_over_ranks(dist, (3.0, 1.5)[rank], "cpu")
        value = bench.job_gflops(2.0e9, 100, world, ms / 1e3)
        out = io.StringIO()
        ref_rc = None
        if rank != 0:
            # the reference arm: ranks other than 0 exit at once, printing nothing
            args = types.SimpleNamespace(workload="2d2048", steps=3, warmup=3)
            with contextlib.redirect_stdout(out):
                ref_rc = bench.run_reference(args)
        dist.barrier()
        q.put((rank, ms, el, value, bench.rank_info(), ref_rc, out.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_the_slowest_and_count_both_replicas():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        results = sorted(q.get(timeout=180) for _ in range(world))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    for rank, ms, el, value, info, ref_rc, printed in results:
        assert ms == 20.0 and el == 3.0  # every rank holds the slowest rank's times
        assert value == pytest.approx(2.0e9 * 100 * world / 0.020 / 1e9)  # both replicas' work
        assert info == (rank, world, rank)
        if rank != 0:
            assert ref_rc == 0 and printed == ""


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(None, 12.5, "cpu") == 12.5
    assert bench.job_gflops(1.0e9, 10, 1, 2.0) == pytest.approx(5.0)
