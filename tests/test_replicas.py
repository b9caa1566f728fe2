"""The bench's multi-GPU form is replicas: each rank solves its own copy of
the workload and the job time is the max over ranks (one scalar all-reduce).
Checked here on CPU with two gloo ranks; the reference arm runs on rank 0
only."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        t = bench.reduce_max(0.5 + rank, world, torch.device("cpu"))

        class A:
            n, steps, warmup = 4, 1, 0
            ref_newton_iters, ref_krylov_iters = 1, 1
        ref = bench.run_reference(A, rank, world) if rank == 1 else "skipped"
        out[rank] = (t, ref)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_max_over_ranks_gloo():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:  # no fork of a process that already runs threads
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == pytest.approx(1.5) and res[1][0] == pytest.approx(1.5)
    assert res[1][1] is None  # the reference arm does no work off rank 0


def test_reference_arm_covers_every_load_step():
    """With fewer timed plus warm-up steps than load steps, the reference
    arm solves the load steps it has not seen (measured, in the order of the
    history), so its value is the sum of five measured load-step times."""
    import math
    import bench

    class A:
        n, steps, warmup = 4, 2, 1

    out = bench.run_reference(A, 0, 1)
    assert math.isfinite(out["value"]) and out["value"] > 0
    assert out["config"]["load_steps_not_timed_as_steps"] == {1: "warm-up", 4: "after the timed steps",
                                                              5: "after the timed steps"}
    assert out["e2e"]["value"] == out["value"] == out["cpu_baseline"]["value"]
