"""The benchmark's multi-rank logic on two gloo ranks (CPU): every rank runs
its own replica (seeds differ, sizes do not), the timing is the slowest
rank's, the rate counts the units of all ranks, and only rank 0 runs the
reference arm.  Batches and served jobs are split over the ranks by the
size-balanced greedy rule (cac_b200.shard), with only metrics gathered."""
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


def _metrics_worker(rank, ws, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from cac_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        units = shard.sum_over_ranks(100.0 * (rank + 1), dist)
        rec = {"lat": [0.5 + rank, 1.0 + rank], "site_steps": 10.0 * (rank + 1), "codes": {"3": 1 + rank},
               "failed": {} if rank == 0 else {"unstable": 1}, "makespan": 2.0 + rank, "jobs": 2}
        parts = shard.gather_objects(rec, dist)
        out.put((rank, units, bench.merge_serving(parts), sum(p["jobs"] for p in parts)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_metrics_only():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_metrics_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, units, (lat, site_steps, codes, failed, makespan), njobs in res:
        assert units == 300.0
        assert sorted(lat) == [0.5, 1.0, 1.5, 2.0]
        assert site_steps == 30.0 and makespan == 3.0 and njobs == 4
        assert codes == {"3": 3} and failed == {"unstable": 1}


def test_balanced_partition_rule():
    sys.path.insert(0, ROOT)
    import random
    from cac_b200 import shard
    rnd = random.Random(5)
    for n, ws in ((37, 2), (256, 8), (5, 8), (0, 3)):
        sizes = [rnd.randint(1, 1000) for _ in range(n)]
        parts = shard.balanced_partition(sizes, ws)
        assert len(parts) == ws
        assert sorted(i for p in parts for i in p) == list(range(n))
        assert parts == shard.balanced_partition(sizes, ws)       # deterministic
        loads = [sum(sizes[i] for i in p) for p in parts]
        if n:
            assert max(loads) <= sum(sizes) / ws + max(sizes)


def test_batch_and_stream_shares_cover_the_global_set():
    """Each rank's share of the 256-per-GPU replica set and of the job
    stream: disjoint, together the whole set, sizes balanced."""
    sys.path.insert(0, ROOT)
    import bench
    from cac_b200 import gen
    ws = 4
    specs = gen.replica_specs(256 * ws, seed=13)
    shares = [bench.batch_share(specs, r, ws) for r in range(ws)]
    assert sorted(i for sh in shares for i in sh) == list(range(256 * ws))
    loads = [sum(specs[i][0] + 8 * specs[i][1] for i in sh) for sh in shares]
    assert max(loads) - min(loads) <= max(sp[0] + 8 * sp[1] for sp in specs)
    assert gen.replica_specs(256, seed=13) == specs[:256]         # one GPU: the same 256 replicas
