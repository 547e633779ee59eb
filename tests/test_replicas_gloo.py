"""The multi-GPU path of the benchmark is replicas only: every rank loads its own seeded replica
circuit, with no data-path exchange, and the whole-job figures are the ranks' summed instances over
the slowest rank's time. This runs that host logic (bench.replica_totals / replica_seed) on two
CPU processes over gloo, as torchrun would launch them."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n = 1000 + 7 * rank          # replica sizes differ with the seed
        ms = 1.5 if rank == 0 else 2.25
        n_all, ms_max = bench.replica_totals(dist, n, ms, "cpu")
        out[rank] = (n_all, ms_max, bench.replica_seed(2026, rank))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_totals_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][:2] == res[1][:2] == (1000 + 1007, 2.25)
    assert res[0][2] != res[1][2]  # each rank loads its own replica


def test_single_process_totals_pass_through():
    import bench

    assert bench.replica_totals(None, 123, 4.5, "cpu") == (123, 4.5)
