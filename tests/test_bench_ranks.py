"""The benchmark's multi-rank plumbing (one replica per GPU under torchrun):
the max-over-ranks timing reduction and the barrier, run as two `gloo`
ranks on the CPU."""

import os
import pathlib
import socket
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(world)
        # each rank's timed region; the job's time is the slowest rank's
        results[rank] = (bench.max_over_ranks(1.0 + 0.25 * rank, world, device="cpu"), bench.max_over_ranks(7.0, 1))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_with_two_gloo_ranks():
    import torch.multiprocessing as mp

    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        results = manager.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, results)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        codes = [p.exitcode for p in procs]
        got = dict(results)
    assert codes == [0, 0], codes
    assert got == {0: (1.25, 7.0), 1: (1.25, 7.0)}

