"""The multi-GPU path of the benchmark without GPUs: independent replicas, one per rank, whose
whole-job figures are the particle-steps of all ranks over the slowest rank's time.  Two
ranks on the gloo backend (127.0.0.1), run as spawned processes."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "op-pic_b200"))
    import torch
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    dev = torch.device("cpu")
    # rank r: (r + 1) * 100 particle-steps in (r + 1) * 2 s, ms per step (r + 1) * 7
    value, ms = bench.replica_job_value((rank + 1) * 100.0, (rank + 1) * 2.0, (rank + 1) * 7.0, dev)
    e2e = bench.replica_sum(10.0 * (rank + 1), dev)
    dist.barrier()
    dist.destroy_process_group()
    Path(out_dir, f"rank{rank}.txt").write_text(f"{value} {ms} {e2e}")


def test_two_gloo_replicas_combine(tmp_path):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        value, ms, e2e = (float(v) for v in (tmp_path / f"rank{r}.txt").read_text().split())
        assert value == pytest.approx((100.0 + 200.0) / 4.0)  # all particle-steps over the slowest rank
        assert ms == pytest.approx(14.0)
        assert e2e == pytest.approx(30.0)


def test_single_process_is_plain_ratio():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.replica_job_value(50.0, 2.0, 3.0, "cpu") == (25.0, 3.0)
    assert bench.replica_sum(4.0, "cpu") == 4.0


def test_reference_arm_other_ranks_do_nothing(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")
    assert bench.arm_reference(None) == {}


def _shard_rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "op-pic_b200"))
    import numpy as np
    import torch
    import torch.distributed as dist

    import bench
    from oppb.advec import shard_instances

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    rng = np.random.default_rng(11)  # the same seeded ensemble on every rank
    sides = rng.integers(64, 513, 64)
    ppcs = rng.integers(10, 201, 64)
    weights = [int(s) * int(s) * int(p) for s, p in zip(sides, ppcs)]
    shards = shard_instances(weights, world)
    seen = [None] * world
    dist.all_gather_object(seen, shards)
    mine = sum(weights[k] for k in shards[rank])
    # each rank's shard "runs" in time proportional to its particles: 1 s per 1e8 particle-steps
    value, _ = bench.replica_job_value(float(mine), mine / 1e8, 1.0, torch.device("cpu"))
    dist.barrier()
    dist.destroy_process_group()
    same = all(x == shards for x in seen)
    Path(out_dir, f"shard{rank}.txt").write_text(f"{int(same)} {value} {sum(weights)} {max(sum(weights[k] for k in x) for x in shards)}")


def test_two_gloo_ranks_split_the_ensemble(tmp_path):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_shard_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        same, value, total, largest = (tmp_path / f"shard{r}.txt").read_text().split()
        assert same == "1"  # both ranks computed the same split
        # all particle-steps over the slowest (most loaded) rank's time
        assert float(value) == pytest.approx(float(total) / (float(largest) / 1e8))
