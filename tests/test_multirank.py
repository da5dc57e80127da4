"""The host logic of multi-GPU runs, on CPU with two gloo ranks: every rank
takes the same collective steps, times reduce by maximum and work by sum
(bench.reduce_over_ranks), and the batched and differentiable workloads give
each rank its own shard of scenes."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from mpm_b200.scenes import create_adjoint_scenes, create_batched_tank_scenes


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        maxima, sums = bench.reduce_over_ranks(dist, "cpu", [1.0 + rank, 10.0 - rank], [100.0 * (rank + 1)])
        out[rank] = (maxima, sums)
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_times_by_maximum_and_work_by_sum():
    world = 2
    port = _free_port()
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        results = dict(out)
    for rank in range(world):
        maxima, sums = results[rank]
        assert maxima == [2.0, 10.0]
        assert sums == [300.0]


def test_single_process_reduces_to_its_own_values():
    import bench
    assert bench.reduce_over_ranks(None, "cpu", [3.0], [4.0]) == ([3.0], [4.0])


def test_rank_shards_are_different_scenes():
    a = create_batched_tank_scenes(3, first=0, particles=(500, 2000), sides=(32, 64))
    b = create_batched_tank_scenes(3, first=3, particles=(500, 2000), sides=(32, 64))
    both = create_batched_tank_scenes(6, first=0, particles=(500, 2000), sides=(32, 64))
    for (p, c), (q, d) in zip(a + b, both):
        assert c == d and np.array_equal(p.px, q.px)
    assert not any(np.array_equal(p.px, q.px) for (p, _), (q, _) in zip(a, b))
    x = create_adjoint_scenes(2, first=0, water_columns=8, water_rows=8, solid_side=4, cells=32)
    y = create_adjoint_scenes(2, first=2, water_columns=8, water_rows=8, solid_side=4, cells=32)
    assert not any(np.array_equal(p.vx, q.vx) for (p, _, _), (q, _, _) in zip(x, y))


def test_scene_specs_match_the_built_scenes():
    from mpm_b200.scenes import batched_tank_scene_specs
    specs = batched_tank_scene_specs(5, first=7, particles=(500, 2000), sides=(32, 64))
    scenes = create_batched_tank_scenes(5, first=7, particles=(500, 2000), sides=(32, 64))
    assert specs == [(len(p.px), c["grid"]["cellsX"]) for p, c in scenes]
    picked = create_batched_tank_scenes(indices=[9, 7], particles=(500, 2000), sides=(32, 64))
    assert np.array_equal(picked[0][0].px, scenes[2][0].px) and np.array_equal(picked[1][0].px, scenes[0][0].px)


def test_cost_shards_cover_every_scene_once_and_balance():
    from mpm_b200.scenes import batched_tank_scene_specs
    from mpm_b200.sharding import scene_cost, shard_by_cost
    for world in (1, 2, 3, 8):
        specs = batched_tank_scene_specs(512 * world)
        costs = [scene_cost(n, s, s) for n, s in specs]
        shares = shard_by_cost(costs, world)
        flat = sorted(k for share in shares for k in share)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[k] for k in share) for share in shares]
        # the longest-processing-time rule: every rank within one scene of the mean
        assert max(loads) - sum(loads) / world <= max(costs)
        assert max(loads) / min(loads) < 1.01
        assert shard_by_cost(costs, world) == shares  # the same split on every rank


def _shard_main(rank, world, port, out):
    from mpm_b200.scenes import batched_tank_scene_specs
    from mpm_b200.sharding import scene_cost, shard_by_cost
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        specs = batched_tank_scene_specs(64 * world, particles=(500, 2000), sides=(32, 64))
        costs = [scene_cost(n, s, s) for n, s in specs]
        mine = shard_by_cost(costs, world)[rank]
        import torch
        load = torch.tensor([float(sum(costs[k] for k in mine)), float(len(mine))])
        gathered = [torch.zeros(2) for _ in range(world)]
        dist.all_gather(gathered, load)
        out[rank] = (mine, [g.tolist() for g in gathered])
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_disjoint_balanced_shares():
    world = 2
    port = _free_port()
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_shard_main, args=(world, port, out), nprocs=world, join=True)
        results = dict(out)
    shares = [set(results[r][0]) for r in range(world)]
    assert not shares[0] & shares[1] and len(shares[0] | shares[1]) == 64 * world
    loads = [v[0] for v in results[0][1]]
    assert max(loads) / min(loads) < 1.02
