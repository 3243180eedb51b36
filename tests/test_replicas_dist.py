"""The multi-GPU form of the path is replicas only (one independent system per
rank; a system does not shard without domain decomposition): bench.py
--gpus N runs one replica per rank, times each on its device and reports the
whole-job rate from the slowest rank.  Its host logic -- the process group,
the barrier, the max over ranks, the aggregation and the per-rank seeds --
runs here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    r, w, local = bench.dist_info()
    dist = bench.init_dist(w, "gloo")
    try:
        ms = 10.0 + 5.0 * r                         # rank 1 is the slow one
        bench.barrier(dist, "cpu")
        ms_max = bench.reduce_max(dist, ms, "cpu")
        value = bench.replicas_value(w, 1000, 20, ms_max)
        bench.barrier(dist, "cpu")
        out.put((r, w, local, ms_max, value))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 and r[2] == r[0] for r in res)
    # every rank sees the slowest rank's time and the same whole-job rate
    assert all(r[3] == 15.0 for r in res)
    assert all(r[4] == pytest.approx(2 * 1000 * 20 / 0.015) for r in res)


def test_one_rank_needs_no_process_group():
    import bench
    assert bench.init_dist(1, "gloo") is None
    assert bench.reduce_max(None, 3.5) == 3.5
    bench.barrier(None)
    assert bench.replicas_value(1, 128000, 40, 1024.0) == pytest.approx(128000 * 40 / 1.024)
