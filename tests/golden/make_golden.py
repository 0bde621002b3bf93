"""Generates the golden fixtures that pin the oracle to the reference.

Runs only where the reference tree is mounted: it drives the reference's own
layer/cuda_bvh_backend.cu, compiled from its sources into oracle/_ref/ by
`make -C oracle ref`, through the reference's C-ABI (cudaBVH_build ->
getStacklessBVH2 / getPackedTris / getNodeData / getTriData / getBounds, and
cudaBVH_buildTLASFast), on small seeded inputs, and stores inputs and
outputs as compressed .npz files next to this script.  The tests then check
the oracle's restatement against these files on any machine.

    python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "vk-rt-cuda-raytracing_b200"))

from oracle import oracle as O  # noqa: E402
from rtb200 import scenes  # noqa: E402


def builder_inputs():
    rs = np.random.RandomState(1234)
    spheres = scenes.scene_spheres_100k(0)[:1002]
    soup = rs.uniform(-10, 10, size=(400, 9)).astype(np.float32)
    # pathological: duplicated triangles, a flat grid, a sliver and a point
    dup = np.tile(np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32), (40, 1))
    g = np.stack(np.meshgrid(np.arange(8), np.arange(8)), -1).reshape(-1, 2).astype(np.float32)
    flat = np.concatenate([np.stack([g[:, 0], np.zeros(64), g[:, 1], g[:, 0] + 1, np.zeros(64), g[:, 1],
                                     g[:, 0], np.zeros(64), g[:, 1] + 1], 1)]).astype(np.float32)
    odd = np.array([[0, 0, 0, 1e-7, 0, 0, 2e-7, 0, 0], [5, 5, 5, 5, 5, 5, 5, 5, 5]], np.float32)
    edge = np.concatenate([dup, flat, odd]).astype(np.float32)
    return {"spheres1002": spheres, "soup400": soup, "edge106": edge}


def main():
    ref = O.RefBackend()
    for name, tris in builder_inputs().items():
        ex = ref.build_exports(tris)
        np.savez_compressed(HERE / f"ref_build_{name}.npz", tris=tris, **ex)
        print(name, tris.shape[0], "dfs nodes", ex["dfs"].size // 8)
    rs = np.random.RandomState(7)
    for n in (1, 2, 3, 64, 1000):
        lo = rs.uniform(-50, 50, size=(n, 3)).astype(np.float32)
        aabbs = np.concatenate([lo, lo + rs.uniform(0.1, 5, size=(n, 3)).astype(np.float32)], 1)
        nodes, ordered = ref.tlas_fast(aabbs)
        np.savez_compressed(HERE / f"ref_tlasfast_{n}.npz", aabbs=aabbs, nodes=nodes, ordered=ordered)
        print("tlas", n, nodes.size // 8)


if __name__ == "__main__":
    main()
