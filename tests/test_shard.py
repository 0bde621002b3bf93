"""Partitioning across GPUs (rtb200.shard) and its use by bench.py's
batched and served forms, on CPU: blocks cover the work exactly once, the
largest scene block is the least any contiguous split achieves, and two gloo
ranks derive the same partition and gather each other's latencies."""
import itertools
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from rtb200 import scenes, shard


@pytest.mark.parametrize("n", [0, 1, 7, 32, 2_000_000, 2_000_003])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_ray_blocks_cover(n, world):
    blocks = [shard.ray_block(n, world, r) for r in range(world)]
    assert blocks[0][0] == 0
    for (f0, c0), (f1, _) in zip(blocks, blocks[1:]):
        assert f0 + c0 == f1
    assert blocks[-1][0] + blocks[-1][1] == n
    counts = [c for _, c in blocks]
    assert max(counts) - min(counts) <= 1


def test_ray_block_rejects_bad_rank():
    with pytest.raises(ValueError):
        shard.ray_block(10, 2, 2)
    with pytest.raises(ValueError):
        shard.ray_block(-1, 2, 0)


def _best_max_load(w, world):
    """Exhaustive least largest block over contiguous splits into <= world blocks."""
    n, best = len(w), None
    for k in range(1, min(world, n) + 1):
        for cuts in itertools.combinations(range(1, n), k - 1):
            b = [0, *cuts, n]
            m = max(sum(w[b[i]:b[i + 1]]) for i in range(k))
            best = m if best is None else min(best, m)
    return best


@pytest.mark.parametrize("seed", range(40))
def test_scene_blocks_optimal_and_nonempty(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 9))
    world = int(rng.integers(1, 5))
    w = [int(x) for x in rng.integers(0, 50, n)]
    b = shard.scene_blocks(w, world)
    assert len(b) == world + 1 and b[0] == 0 and b[-1] == n
    assert all(x <= y for x, y in zip(b, b[1:]))
    loads = [sum(w[b[i]:b[i + 1]]) for i in range(world)]
    assert max(loads) == _best_max_load(w, world)
    if n >= world:
        assert all(b[i + 1] > b[i] for i in range(world))


def test_owner_and_requests_partition():
    b = shard.scene_blocks([5, 1, 1, 9, 2, 2, 7, 1], 3)
    scene = np.array([0, 3, 7, 2, 6, 6, 1, 4, 5, 0])
    own = shard.owner_of(b, scene)
    for r in range(3):
        sel = shard.requests_for_rank(scene, b, r)
        assert (own[sel] == r).all() and (np.diff(sel) > 0).all()
    assert sum(len(shard.requests_for_rank(scene, b, r)) for r in range(3)) == scene.size
    with pytest.raises(ValueError):
        shard.owner_of(b, [8])


def test_batched_partition_balances_build_work():
    ntri, nray = scenes.batched_sizes()
    w = ntri + nray // 20
    for world in (2, 4, 8):
        b = shard.scene_blocks(w, world)
        loads = np.array([w[b[i]:b[i + 1]].sum() for i in range(world)])
        assert loads.sum() == w.sum()
        assert loads.max() <= w.sum() / world + w.max()  # within one scene of an even split


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        # the served form's partition, as bench.served_legs derives it on each rank
        _, scene0, nray0, _, _ = scenes.served_trace(bench.SERVED_NREQ, rate=bench.SERVED_RATE)
        b = shard.scene_blocks(np.bincount(scene0, weights=nray0, minlength=16).astype(np.int64), ws)
        sel = shard.requests_for_rank(scene0, b, rank)
        lat = 10.0 * rank + np.arange(sel.size, dtype=np.float64)  # stand-in per-request latencies
        all_sel = bench.gather_over_ranks(sel, ws)
        all_lat = bench.gather_over_ranks(lat, ws)
        span = float(bench.gather_over_ranks([1.5 + rank], ws).max())
        out.put((rank, b, all_sel.tolist(), all_lat.tolist(), span))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_partition_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    (_, b0, sel0, lat0, span0), (_, b1, sel1, lat1, span1) = res
    assert b0 == b1                                   # both ranks derive the same scene blocks
    assert sel0 == sel1 and lat0 == lat1              # and gather the same arrays, in rank order
    assert sorted(sel0) == list(range(256))           # every request served by exactly one rank
    assert span0 == span1 == 2.5                      # the slowest rank's span
