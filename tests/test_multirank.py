"""The benchmark's multi-rank logic on two gloo ranks (CPU): every rank runs
its own replica (seeds differ, sizes do not), the timing is the slowest
rank's, the rate counts the units of all ranks, and only rank 0 runs the
reference arm."""
import io
import os
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, ws, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        ms = 10.0 + 5.0 * rank                       # rank 1 is the slower one
        slowest = bench.max_over_ranks(ms, dist)
        rate = bench.whole_job_rate(1000, 20, ws, slowest / 1000.0)
        seed = bench.rank_seed(2, rank)

        class Args:
            workload, steps, warmup, gpus = "lj_small", 1, 0, ws
        buf = io.StringIO()
        with redirect_stdout(buf):
            if rank != 0:
                bench.reference_arm(Args, rank, ws)   # must return at once, silently
        dist.barrier()
        out.put((rank, slowest, rate, seed, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, rate0, seed0, out0), (r1, s1, rate1, seed1, out1) = res
    assert s0 == s1 == 15.0
    assert rate0 == rate1 == pytest.approx(1000 * 20 * 2 / 0.015)
    assert seed0 != seed1
    assert out1 == ""


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.whole_job_rate(10, 4, 1, 2.0) == 20.0
