"""The multi-rank plumbing of bench.py on CPU: two gloo ranks, as torchrun
starts them, each with its own device time; the job's time is the slowest
rank's and the ensemble rate counts every rank's steps.  Also: only rank 0 of
the reference arm does work."""
import json
import os
import socket
import tempfile

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        my_ms = 100.0 + 50.0 * rank                 # rank 1 is the slower one
        max_ms = bench.max_over_ranks(my_ms, world, dist, torch, "cpu")
        rate = bench.ensemble_rate(10, max_ms, world)
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max_ms": max_ms, "rate": rate}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_ensemble_rate_gloo():
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(world, _free_port(), d), nprocs=world, start_method="spawn")
        res = [json.load(open(os.path.join(d, f"rank{r}.json"))) for r in range(world)]
    for r in res:
        assert r["max_ms"] == 150.0                 # every rank agrees on the slowest rank's time
        assert r["rate"] == pytest.approx(2 * 10 / 0.150)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(12.5, 1, None, torch, "cpu") == 12.5
    assert bench.ensemble_rate(10, 500.0, 1) == pytest.approx(20.0)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    class Args:
        lmax, nr, warmup, steps, gpus = 15, 16, 0, 1, 2
    bench.run_reference(Args, rank=1)               # no work, no output on other ranks
    assert capsys.readouterr().out == ""
