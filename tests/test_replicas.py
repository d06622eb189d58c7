"""The multi-GPU form of the path on the CPU: two `gloo` ranks.

Each rank takes its slice of one Philox population, generates its geometries
with the host twin of the device sampler, and times "its work"; the job's rate
uses the max over ranks. The slices are disjoint, cover the population, and are
bit-identical to the same sims generated by a single process; the reference arm
does no work on ranks other than 0.
"""
from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT

S_PER_RANK = 512


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import datetime

    import torch
    import torch.distributed as dist

    from pkg_loader import load_submodule

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    rp = load_submodule("replicas")
    sp = load_submodule("sampling")
    wl = load_submodule("workloads")
    first, count = rp.shard(rank, world, S_PER_RANK)
    pos, _, flags = sp.sample_ball_host(wl.CH4, count, seed=99, first_sim=first)
    assert not flags.any()
    fake_ms = 10.0 + rank  # rank 1 is the slowest
    mx = rp.max_over_ranks(fake_ms)
    rate = rp.aggregate_rate(world, count, 3, mx)
    gathered = [torch.zeros((count, 5, 3), dtype=torch.float32) for _ in range(world)]
    dist.all_gather(gathered, torch.from_numpy(pos))
    if rank == 0:
        np.savez(os.path.join(out_dir, "replicas.npz"), pos=torch.cat(gathered).numpy(), mx=mx, rate=rate,
                 first=np.array([rp.shard(r, world, S_PER_RANK)[0] for r in range(world)]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_sample_and_reduce(ce, wl, tmp_path):
    sp = pytest.importorskip("coulomb_explosion_b200.sampling")
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    z = np.load(tmp_path / "replicas.npz")
    assert float(z["mx"]) == 11.0
    assert float(z["rate"]) == pytest.approx(world * S_PER_RANK * 3 / 11e-3)
    assert list(z["first"]) == [0, S_PER_RANK]
    single, _, _ = sp.sample_ball_host(wl.CH4, world * S_PER_RANK, seed=99, first_sim=0)
    assert np.array_equal(z["pos"], single)


def test_reference_arm_does_no_work_off_rank_zero(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        steps, warmup = 1, 1

    assert bench.run_reference_arm(A()) == 0


def test_shard_arguments():
    from pkg_loader import load_submodule

    rp = load_submodule("replicas")
    assert rp.shard(3, 4, 10) == (30, 10)
    with pytest.raises(ValueError):
        rp.shard(4, 4, 10)
    assert rp.max_over_ranks(2.5) == 2.5
