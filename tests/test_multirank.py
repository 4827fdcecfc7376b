"""The N>1 bench path on CPU: two gloo ranks (127.0.0.1) take the same
replica batch, reduce the step time to the slowest rank's and report the
whole-job rate; the reference arm runs on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        spec = bench.batch_spec()
        key = [(s["dims"], s["mass"], s["eps"], s["nrhs"], s["gauge_seed"], s["rhs_seed"]) for s in spec]
        keys = [None] * world
        dist.all_gather_object(keys, key)
        ms = bench.max_over_ranks(100.0 + 10.0 * rank, world, device="cpu")
        total = sum(s["nrhs"] for s in spec)
        out[rank] = (keys[0] == keys[1], ms, bench.replica_value(world, total, ms), total)
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    assert sorted(out.keys()) == [0, 1]
    for r in range(world):
        same, ms, value, total = out[r]
        assert same  # replicas: every rank solves the identical seeded batch
        assert ms == 110.0  # the slowest rank's step time, on every rank
        assert value == pytest.approx(world * total / 0.110)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")

    class Args:
        warmup, steps, gpus, ref_budget = 1, 1, 2, 1.0
    bench.run_reference_arm(Args(), bench.batch_spec())
    assert capsys.readouterr().out == ""
