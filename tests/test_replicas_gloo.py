"""Multi-GPU is replicas only (no data exchange). The host-side plumbing that
bench.py uses under torchrun -- process group, barrier, max over ranks of the
timed region, whole-job throughput -- runs here as two gloo ranks on the CPU."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup(world, backend="gloo")
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    slowest = bench.barrier_max(1.0 + rank, w)      # rank r "took" 1 + r seconds
    rate = bench.job_throughput(w, 1e9, 10, slowest)
    out.put((rank, slowest, rate))
    dist.destroy_process_group()


def test_two_rank_max_and_throughput():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, rate in res:
        assert slowest == 2.0                      # the max over ranks, on every rank
        assert rate == pytest.approx(2 * 1e9 * 10 / 2.0 / 1e9)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.barrier_max(3.5, 1) == 3.5
    assert bench.job_throughput(1, 2e9, 5, 2.0) == pytest.approx(5.0)
