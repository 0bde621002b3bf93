"""Philox4x32-10 counter-based RNG in numpy (Salmon, Moraes, Dror, Shaw,
"Parallel random numbers: as easy as 1, 2, 3", SC'11).

Used to draw seeded synthetic scenes and rays.  Key = (seed, stream id),
counter = (item, draw, 0, 0).  The CUDA path tracer evaluates the same
function on the device (csrc/rt_common.cuh), so host and device streams agree.
"""
from __future__ import annotations

import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
W0 = np.uint32(0x9E3779B9)
W1 = np.uint32(0xBB67AE85)
MASK32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr: np.ndarray, key: np.ndarray) -> np.ndarray:
    """ctr: (N, 4) uint32, key: (2,) or (N, 2) uint32 -> (N, 4) uint32."""
    ctr = np.asarray(ctr, dtype=np.uint32)
    key = np.asarray(key, dtype=np.uint32)
    c0, c1, c2, c3 = (ctr[:, i].astype(np.uint64) for i in range(4))
    if key.ndim == 1:
        k0 = np.full(ctr.shape[0], key[0], dtype=np.uint64)
        k1 = np.full(ctr.shape[0], key[1], dtype=np.uint64)
    else:
        k0 = key[:, 0].astype(np.uint64)
        k1 = key[:, 1].astype(np.uint64)
    for _ in range(10):
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK32
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
        k0 = (k0 + np.uint64(W0)) & MASK32
        k1 = (k1 + np.uint64(W1)) & MASK32
    return np.stack([c0, c1, c2, c3], axis=1).astype(np.uint32)


def u01(bits: np.ndarray) -> np.ndarray:
    """uint32 -> float32 in [0, 1) with 24 random bits (exact in fp32)."""
    return ((bits >> np.uint32(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)).astype(np.float32)


def uniforms(seed: int, stream: int, n: int, draws: int = 4) -> np.ndarray:
    """(n, draws) float32 uniforms for items 0..n-1 of one (seed, stream)."""
    blocks = (draws + 3) // 4
    out = np.empty((n, blocks * 4), dtype=np.float32)
    key = np.array([seed & 0xFFFFFFFF, stream & 0xFFFFFFFF], dtype=np.uint32)
    items = np.arange(n, dtype=np.uint64)
    for b in range(blocks):
        ctr = np.zeros((n, 4), dtype=np.uint32)
        ctr[:, 0] = (items & MASK32).astype(np.uint32)
        ctr[:, 1] = b
        ctr[:, 2] = (items >> np.uint64(32)).astype(np.uint32)
        out[:, 4 * b: 4 * b + 4] = u01(philox4x32_10(ctr, key))
    return out[:, :draws]
