"""Multi-rank host logic on CPU (gloo, world size 2): ragged scenes are split
over ranks with no overlap and no loss, each rank packs only its share, and
the whole-job figures sum work and take the slowest rank's time."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from flatworld_b200 import shard

N_SCENES = 24


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist

    import flatworld_b200 as fw
    from flatworld_b200.world import PackedWorld, SceneLayout
    from tests import scenes

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        population = [scenes.ragged_batch_one(fw, i, seed=5) for i in range(N_SCENES)]
        weights = [d[1].nelements for d in population]
        mine = shard.share(weights, rank, world)
        packed = PackedWorld([SceneLayout(population[i], dt=5e-5, useAdapativeDT=False) for i in mine])
        assert packed.E == sum(weights[i] for i in mine)
        # every rank sees every other rank's share: disjoint, complete
        got = [None] * world
        dist.all_gather_object(got, mine)
        flat = sorted(i for s in got for i in s)
        assert flat == list(range(N_SCENES)), flat
        # whole-job figures: work summed, time = slowest rank
        local_ms = 10.0 + 5.0 * rank
        total, ms = shard.aggregate(packed.E * 100, local_ms)
        assert total == 100 * sum(weights)
        assert ms == 10.0 + 5.0 * (world - 1)
        loads = torch.tensor([float(packed.E)])
        dist.all_reduce(loads, op=dist.ReduceOp.MAX)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{len(mine)} {packed.E} {float(loads.item())}\n")
    finally:
        dist.destroy_process_group()


def test_partition_is_balanced_deterministic_and_complete():
    rng = np.random.default_rng(0)
    w = rng.integers(100, 20000, size=2048)
    for world in (1, 2, 3, 8):
        parts = shard.partition(w, world)
        assert parts == shard.partition(w, world)
        assert sorted(i for p in parts for i in p) == list(range(len(w)))
        assert all(p == sorted(p) for p in parts)
        loads = [int(w[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= int(w.max())  # LPT bound
    assert shard.partition([5, 5, 5], 2) == [[0, 2], [1]]


def test_aggregate_without_process_group_is_local():
    assert shard.aggregate(7.0, 3.5) == (7.0, 3.5)


@pytest.mark.timeout(240)
def test_two_ranks_shard_pack_and_aggregate(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rows = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(world)]
    assert sum(int(r[0]) for r in rows) == N_SCENES
    assert all(float(r[2]) == max(int(x[1]) for x in rows) for r in rows)
