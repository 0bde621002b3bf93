"""Work partitioning across GPUs: one process per GPU, each with its own
resident copy of the structures it traces, and no exchange on the data path.

Rays are independent and a ray's only output is its own hit record, so the
single-scene trace splits into contiguous ray blocks over replicas of the
BVH; the batched and served forms split whole scenes (and with them every
ray batch and request against those scenes) into contiguous scene blocks
balanced by their work.  The reference traces on one device
(layer/cuda_bvh_backend.cu:1379-1497 is its per-call path); these are the
partitions its path allows.
"""
from __future__ import annotations

import numpy as np


def ray_block(n: int, world: int, rank: int) -> tuple[int, int]:
    """(first, count) of rank's contiguous block of n rays; the first
    n % world ranks take one ray more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n < 0:
        raise ValueError("negative ray count")
    q, r = divmod(n, world)
    first = rank * q + min(rank, r)
    return first, q + (1 if rank < r else 0)


def _blocks_needed(w: np.ndarray, cap: int) -> int:
    blocks, load = 1, 0
    for x in w:
        if load + x > cap:
            blocks += 1
            load = 0
        load += int(x)
    return blocks


def scene_blocks(weights, world: int) -> list[int]:
    """Boundaries b[0] = 0 <= b[1] <= ... <= b[world] = len(weights) of
    contiguous scene blocks, rank r taking scenes b[r] .. b[r+1]-1.  The
    largest block weight is the least any contiguous split achieves (binary
    search on it with a greedy feasibility check); when there are at least
    as many scenes as ranks, every rank gets one or more scenes."""
    w = np.asarray(weights, dtype=np.int64)
    if w.ndim != 1 or (w < 0).any():
        raise ValueError("weights must be a 1-D array of non-negative integers")
    if world < 1:
        raise ValueError("world must be >= 1")
    n = int(w.size)
    if n == 0:
        return [0] * (world + 1)
    lo, hi = int(w.max()), int(w.sum())
    while lo < hi:
        mid = (lo + hi) // 2
        if _blocks_needed(w, mid) <= world:
            hi = mid
        else:
            lo = mid + 1
    cap = lo
    bounds, load = [0], 0
    for i in range(n):
        left_scenes, left_ranks = n - i, world - (len(bounds) - 1)
        # close the block when it would overflow, or when every later rank
        # still needs a scene of its own
        must_close = load > 0 and (load + int(w[i]) > cap or left_scenes <= left_ranks - 1)
        if must_close and len(bounds) < world:
            bounds.append(i)
            load = 0
        load += int(w[i])
    while len(bounds) < world:
        bounds.append(n)
    bounds.append(n)
    return bounds


def owner_of(bounds, scene) -> np.ndarray:
    """Rank that owns each scene id under scene_blocks' boundaries."""
    b = np.asarray(bounds)
    s = np.asarray(scene)
    if ((s < 0) | (s >= b[-1])).any():
        raise ValueError("scene id outside the partition")
    return np.searchsorted(b, s, side="right") - 1


def requests_for_rank(scene_of_request, bounds, rank: int) -> np.ndarray:
    """Indices (in arrival order) of the requests whose scene rank owns."""
    return np.nonzero(owner_of(bounds, scene_of_request) == rank)[0]
