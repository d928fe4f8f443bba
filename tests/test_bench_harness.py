"""bench.py's replica harness on CPU ranks (gloo, world size 2, 127.0.0.1): the
timed region's duration is the maximum over ranks and reaches every rank, the
whole-job value is world x per-rank units over that time, and the reference
arm runs on rank 0 only (the other ranks return without work).  The data path
has no collective: each rank runs its own replica of the workload."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        value = bench.replica_value(1000.0, ms, world)
        ref = bench.run_reference(None, rank, world) if rank != 0 else "skipped"
        dist.barrier()
        q.put((rank, ms, value, ref))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_value_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value, ref in out:
        assert ms == pytest.approx(15.0)              # the slowest rank's time, on every rank
        assert value == pytest.approx(2 * 1000.0 / 15e-3)
    assert out[1][3] is None                          # the reference arm: rank 1 does nothing


def test_single_rank_helpers():
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_value(10.0, 2.0, 1) == pytest.approx(5000.0)
