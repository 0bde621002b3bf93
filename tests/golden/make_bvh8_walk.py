"""Writes two fixtures on a B200, each the engine's 8-wide nodes and
triangle records for a seeded scene, two ray sets, and what the kernels
returned for them -- closest hits, occlusion flags, and the per-ray node
visits and triangle tests of cudaBVH_traceCounters (the counts bench.py
turns into algorithmic bytes per ray):
  bvh8_walk_2k.npz           2,000 triangles, 512 primary + 512 diffuse rays;
  bvh8_walk_3k_diffuse.npz   3,000 triangles in ~75 meshes of 20-60 packed in
                             a 10-unit box, 1,536 diffuse rays leaving their
                             surfaces (incoherent; over half hit, deeper walks).
Each fixture also records the kernel's walk shape (node visits per round,
pending triangle sets).  tests/test_oracle_bvh8.py replays the walks over
the same nodes with the oracle at that shape on the CPU and must reproduce
every value exactly.

    python tests/golden/make_bvh8_walk.py [OUTDIR]   # needs the built library and a GPU
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "vk-rt-cuda-raytracing_b200"))

import torch  # noqa: E402
from cuda.bindings import runtime as cudart  # noqa: E402

from rtb200 import lib, scenes  # noqa: E402
from rtb200.scenes import HIT_DTYPE, RAY_DTYPE  # noqa: E402

NODE_BYTES, REC_BYTES = 80, 48
# the release kernel's walk shape (RTB_NODE_ITERS, RTB_TWO_SETS + 1)
NITERS, SETS = 4, 2
OUT = HERE


def d2h(ptr: int, nbytes: int) -> np.ndarray:
    out = np.empty(nbytes, np.uint8)
    (err,) = cudart.cudaMemcpy(out.ctypes.data, ptr, nbytes, cudart.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == cudart.cudaError_t.cudaSuccess, err
    return out


def run(bvh, rays: np.ndarray, any_hit: bool):
    n = rays.shape[0]
    d_rays = torch.from_numpy(np.ascontiguousarray(rays).view(np.uint8).copy()).cuda()
    d_cnt = torch.zeros(n * 2, dtype=torch.int32, device="cuda")
    bvh.counters(d_rays, n, d_cnt, any_hit=any_hit)
    if any_hit:
        d_out = torch.zeros(n, dtype=torch.uint8, device="cuda")
        bvh.any(d_rays, n, d_out)
    else:
        d_out = torch.zeros(n * 16, dtype=torch.uint8, device="cuda")
        bvh.closest(d_rays, n, d_out)
    torch.cuda.synchronize()
    cnt = d_cnt.cpu().numpy().view(np.uint32).reshape(n, 2)
    out = d_out.cpu().numpy()
    return cnt, (out if any_hit else out.view(HIT_DTYPE))


def fixture(name: str, tris: np.ndarray, rays: np.ndarray):
    bvh = lib.BVH(tris)
    bvh.validate()
    pn, n_nodes, pt, n_recs = bvh.layout()
    nodes = d2h(pn, n_nodes * NODE_BYTES).view(np.uint32).reshape(n_nodes, 20)
    recs = d2h(pt, n_recs * REC_BYTES).view(np.float32).reshape(n_recs, 12)
    cnt_c, hits = run(bvh, rays, False)
    # any hit: the same rays cut short of their closest hit (unoccluded) or
    # past it (occluded), misses left unbounded
    shadow = rays.copy()
    hit = hits["prim"] >= 0
    cut = np.where(np.arange(rays.shape[0]) % 2 == 0, np.float32(0.999), np.float32(1.001))
    shadow["tmax"] = np.where(hit, hits["t"] * cut, np.float32(np.inf)).astype(np.float32)
    cnt_a, occ = run(bvh, shadow, True)
    bvh.close()
    np.savez_compressed(os.path.join(OUT, name), niters=np.int32(NITERS), sets=np.int32(SETS), nodes=nodes, recs=recs,
                        rays=rays.view(np.float32).reshape(-1, 8), hits=hits.view(np.float32).reshape(-1, 4),
                        counts_closest=cnt_c, shadow=shadow.view(np.float32).reshape(-1, 8), occ=occ,
                        counts_any=cnt_a)
    print(f"{name}: {n_nodes} nodes, {n_recs} records, {rays.shape[0]} rays: hit {hit.mean():.2f}, "
          f"occluded {occ.mean():.2f}, nodes/ray {cnt_c[:, 0].mean():.2f} (max {cnt_c[:, 0].max()}), "
          f"tris/ray {cnt_c[:, 1].mean():.2f}")


def main():
    global OUT
    if len(sys.argv) > 1:
        OUT = sys.argv[1]
        os.makedirs(OUT, exist_ok=True)
    torch.cuda.set_device(0)
    tris = scenes.scene_meshes(11, 2000)
    fixture("bvh8_walk_2k.npz", tris, scenes.scene_rays(tris, 1024, seed=5))
    tris = scenes.scene_meshes(12, 3000, box=10.0, lo=20, hi=60)
    fixture("bvh8_walk_3k_diffuse.npz", tris, scenes.scene_rays(tris, 3072, seed=6)[1536:])


if __name__ == "__main__":
    main()
