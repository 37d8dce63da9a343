"""Multi-rank replica bookkeeping on CPU: two gloo ranks stand in for two
GPUs running independent solves (the bench's N > 1 path).  No GPU needed."""

from __future__ import annotations

import importlib
import os
import socket

import pytest

replicas = importlib.import_module("3d_mpi_test_b200.replicas")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out: str) -> None:
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g = replicas.ReplicaGroup(dist, "cpu")
        g.barrier()
        local_ms = 10.0 * (rank + 1)  # rank 1 is the slow replica
        worst = g.max_over_ranks(local_ms)
        gcell = g.throughput(cells_per_rank=1_000_000, steps=100, local_ms=local_ms)
        mine = replicas.shard(list(range(11)), g.rank, g.world)
        g.barrier()
        with open(os.path.join(out, f"rank{rank}.txt"), "w") as f:
            f.write(f"{g.world} {worst} {gcell} {','.join(map(str, mine))}\n")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica(tmp_path):
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, start_method="spawn")
    rows = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(world)]
    items = []
    for w, worst, gcell, mine in rows:
        assert int(w) == world
        assert float(worst) == 20.0
        # 2 ranks x 1e6 cells x 100 steps in 20 ms (the slower rank)
        assert float(gcell) == pytest.approx(2 * 1e6 * 100 / 20e-3 / 1e9)
        items += [int(x) for x in mine.split(",") if x]
    assert sorted(items) == list(range(11))


def test_single_rank_without_process_group():
    g = replicas.ReplicaGroup(None)
    assert (g.world, g.rank) == (1, 0)
    g.barrier()
    assert g.max_over_ranks(3.5) == 3.5
    assert g.throughput(1000, 10, 1.0) == pytest.approx(1000 * 10 / 1e-3 / 1e9)
    with pytest.raises(ValueError):
        g.throughput(1000, 10, 0.0)
    with pytest.raises(ValueError):
        replicas.shard([1, 2], 2, 2)
