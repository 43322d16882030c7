"""The bench's multi-rank plumbing on the CPU: two gloo ranks (127.0.0.1) through dist_setup,
barrier and max_over_ranks, and the replica aggregation rule (the slowest rank's time, every
replica's simulated time counted).  No GPU: the path has no data exchange, so this is all the
N > 1 code that differs from N = 1."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    w, r, local, pg = bench.dist_setup(None)
    assert (w, r, local) == (world, rank, rank) and pg is not None
    bench.barrier(pg)
    t = bench.max_over_ranks(pg, 10.0 + rank)  # rank 1 is the slower replica
    out[rank] = (t, bench.replica_value(200, t, w))
    pg.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    t, value = res[0]
    assert t == 11.0
    import bench
    assert value == pytest.approx(2 * bench.ns_per_day(200 / 0.011))


def test_single_rank_needs_no_process_group():
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    assert bench.dist_setup(None) == (1, 0, 0, None)
    assert bench.max_over_ranks(None, 3.5) == 3.5
