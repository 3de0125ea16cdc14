"""The multi-GPU path of bench.py (--gpus N under torchrun) is independent replicas: each rank
solves its own right-hand sides, ranks meet at a barrier around the timed region, and the
job's time is the slowest rank's. These steps run here as two gloo ranks on the CPU
(world size 2, rendezvous on 127.0.0.1), with no GPU."""

import os
import queue
import socket

import pytest

WORLD = 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(WORLD), LOCAL_RANK=str(rank))
    import bench

    world, r, _ = bench.dist_setup("gloo")
    try:
        seeds = bench.replica_seeds(1, r, 23)
        bench.barrier(world)
        slowest = bench.max_over_ranks(10.0 * (r + 1), world, "cpu")
        bench.barrier(world)
        out.put((r, world, seeds, slowest))
    finally:
        bench.dist_teardown(world)


def test_two_gloo_replicas():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, out)) for r in range(WORLD)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(WORLD):
            r, world, seeds, slowest = out.get(timeout=180)
            got[r] = (world, seeds, slowest)
    except queue.Empty:
        pytest.fail("a gloo rank did not report within 180 s")
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert sorted(got) == [0, 1]
    # every rank sees the slowest rank's time; the right-hand-side streams are disjoint
    assert all(world == WORLD and slowest == 20.0 for world, _, slowest in got.values())
    assert not set(got[0][1]) & set(got[1][1])
    assert len(set(got[0][1])) == 23


def test_single_process_needs_no_process_group():
    import bench

    os.environ.pop("WORLD_SIZE", None)
    world, rank, local = bench.dist_setup("gloo")
    assert (world, rank, local) == (1, 0, 0)
    assert bench.max_over_ranks(3.5, world, "cpu") == 3.5
    bench.barrier(world)
    bench.dist_teardown(world)
