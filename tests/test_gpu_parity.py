"""GPU parity: the CUDA path through the C-ABI against the CPU oracle.

Bar: hit primitive (and instance) ids, t, u, v bit-identical to the oracle
(both evaluate Moller-Trumbore of layer/cuda_bvh_backend.cu:143-157 in exact
IEEE single precision, ties toward the lower id); any-hit flags identical.
"""
import numpy as np
import pytest

from oracle import oracle as O
from rtb200 import lib, scenes
from rtb200.scenes import HIT_DTYPE, RAY_DTYPE

pytestmark = pytest.mark.gpu


def _dev(torch, arr):
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).copy()).cuda()


def gpu_closest(bvh, rays):
    import torch
    d_rays = _dev(torch, rays)
    d_hits = torch.empty(rays.shape[0] * 16, dtype=torch.uint8, device="cuda")
    bvh.closest(d_rays, rays.shape[0], d_hits)
    torch.cuda.synchronize()
    return d_hits.cpu().numpy().view(HIT_DTYPE)


def gpu_any(bvh, rays):
    import torch
    d_rays = _dev(torch, rays)
    d_occ = torch.empty(rays.shape[0], dtype=torch.uint8, device="cuda")
    bvh.any(d_rays, rays.shape[0], d_occ)
    torch.cuda.synchronize()
    return d_occ.cpu().numpy()


def assert_hits_equal(a, b, what=""):
    bad = np.nonzero((a["prim"] != b["prim"]) | (a["t"].view(np.uint32) != b["t"].view(np.uint32)) |
                     (a["u"].view(np.uint32) != b["u"].view(np.uint32)) |
                     (a["v"].view(np.uint32) != b["v"].view(np.uint32)))[0]
    assert bad.size == 0, f"{what}: {bad.size} rays differ, first {bad[:5]}: {a[bad[:3]]} vs {b[bad[:3]]}"


@pytest.fixture(scope="module")
def small_scene():
    return scenes.scene_spheres_100k(0)[:3002]


def test_closest_and_any_small_vs_brute_force(cuda, small_scene):
    bvh = lib.BVH(small_scene)
    rays = scenes.random_rays(5, 20000)
    ref = O.brute_closest(small_scene, rays)
    assert_hits_equal(gpu_closest(bvh, rays), ref, "device")
    assert_hits_equal(bvh.closest_host(rays), ref, "host")
    occ = O.brute_any(small_scene, rays)
    assert np.array_equal(gpu_any(bvh, rays), occ)
    assert np.array_equal(bvh.any_host(rays), occ)
    assert (ref["prim"] >= 0).mean() > 0.2


def test_primary_1080p_100k_every_ray(cuda):
    """Primary-ray workload: 100,002 triangles, 1920x1080 pinhole rays; every ray checked."""
    tris = scenes.scene_spheres_100k(0)
    bvh = lib.BVH(tris)
    rays = scenes.primary_1080p()
    ob = O.OracleBVH(tris, nbins=32, max_leaf=4)
    ref = ob.closest(rays)
    got = gpu_closest(bvh, rays)
    assert_hits_equal(got, ref, "primary 1080p")
    assert 0.2 < (ref["prim"] >= 0).mean() < 0.95


def test_incoherent_rays_vs_oracle(cuda):
    """Incoherent-ray workload shape on a 400K-triangle scene: cosine diffuse bounces
    (closest hit) and area-light shadow rays (any hit) from primary hits."""
    tris = scenes.scene_meshes(1, 400_000)
    bvh = lib.BVH(tris)
    prim = scenes.pinhole_rays(480, 270, scenes.CAM_EYE, scenes.CAM_TARGET)
    ph = gpu_closest(bvh, prim)
    p, nrm = scenes.hit_frame(tris, prim, ph)
    dif = scenes.diffuse_rays(p, nrm, 200_000, seed=3)
    sha = scenes.shadow_rays(p, nrm, 200_000, seed=4)
    ob = O.OracleBVH(tris, nbins=32, max_leaf=4)
    assert_hits_equal(ob.closest(prim), ph, "primary")
    assert_hits_equal(gpu_closest(bvh, dif), ob.closest(dif), "diffuse")
    assert np.array_equal(gpu_any(bvh, sha), ob.any(sha))


def test_edge_cases(cuda):
    # axis-aligned box faces, a flat grid, zero-area and duplicate triangles
    box = scenes.box_mesh(3) * 2.0
    flat = scenes.ground_plane(-3.0, 4.0)
    degen = np.array([[[0, 0, 0], [0, 0, 0], [0, 0, 0]], [[1, 1, 1], [2, 2, 2], [3, 3, 3]]], np.float64)
    dup = np.repeat(scenes.ground_plane(5.0, 2.0)[:1], 3, axis=0)
    tris = np.concatenate([box, flat, degen, dup]).reshape(-1, 9).astype(np.float32)
    bvh = lib.BVH(tris)
    rs = np.random.RandomState(0)
    n = 4000
    rays = np.zeros(n, RAY_DTYPE)
    rays["org"] = rs.uniform(-6, 6, (n, 3)).astype(np.float32)
    d = rs.normal(size=(n, 3))
    # axis-aligned and zero-component directions
    d[: n // 4] = np.eye(3)[rs.randint(0, 3, n // 4)] * rs.choice([-1, 1], (n // 4, 1))
    d[n // 4: n // 2, rs.randint(0, 3)] = 0.0
    rays["dir"] = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    rays["tmin"] = 0.0
    rays["tmax"] = rs.choice([1e30, 3.0], n).astype(np.float32)
    # rays starting exactly on faces
    rays["org"][-200:, 0] = 2.0
    # NaN direction: never hits
    rays["dir"][-1] = np.nan
    ref = O.brute_closest(tris, rays)
    assert_hits_equal(gpu_closest(bvh, rays), ref, "edge")
    assert np.array_equal(gpu_any(bvh, rays), O.brute_any(tris, rays))
    assert ref["prim"][-1] == -1
    # a hit exactly at tmax is rejected, just beyond it accepted
    r1 = np.zeros(2, RAY_DTYPE)
    r1["org"] = (3.5, 10.0, 3.5)  # above the y = -3 plane, clear of the box and the y = 5 plane
    r1["dir"] = (0, -1, 0)
    r1["tmax"] = (13.0, np.nextafter(np.float32(13.0), np.float32(1e30)))
    h = bvh.closest_host(r1)
    assert h["prim"][0] == -1 and h["prim"][1] >= 0 and h["t"][1] == 13.0


def test_single_triangle_and_zero_rays(cuda):
    tri = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32)
    bvh = lib.BVH(tri)
    r = np.zeros(3, RAY_DTYPE)
    r["org"] = [(0.2, 0.2, 1), (2, 2, 1), (0.2, 0.2, -1)]
    r["dir"] = [(0, 0, -1), (0, 0, -1), (0, 0, 1)]
    r["tmax"] = 1e30
    h = bvh.closest_host(r)
    assert h["prim"].tolist() == [0, -1, 0]
    assert np.allclose(h["t"][[0, 2]], 1.0)
    assert bvh.closest_host(np.zeros(0, RAY_DTYPE)).shape == (0,)


def test_reference_shaped_entry_points(cuda, small_scene):
    bvh = lib.BVH(small_scene)
    side = 256
    cam = (0.0, 0.0, -80.0)
    mrs, t = bvh.trace_primary(side, cam)
    assert mrs > 0
    # the same square camera in float32 on the host (layer/cuda_bvh_backend.cu:69-74)
    px = (np.arange(side * side) % side).astype(np.float32)
    py = (np.arange(side * side) // side).astype(np.float32)
    u = (px + np.float32(0.5)) / np.float32(side) * np.float32(2) - np.float32(1)
    v = (py + np.float32(0.5)) / np.float32(side) * np.float32(2) - np.float32(1)
    rl = np.float32(1) / np.sqrt(u * u + v * v + np.float32(1))
    rays = np.zeros(side * side, RAY_DTYPE)
    rays["org"] = cam
    rays["dir"] = np.stack([u * rl, v * rl, rl], 1)
    rays["tmax"] = 1e30
    ref = O.brute_closest(small_scene, rays)
    exp_t = np.where(ref["prim"] >= 0, ref["t"], np.float32(1e30))
    assert np.array_equal(t.view(np.uint32), exp_t.view(np.uint32))
    # traceDiffuse: host SoA rays in caller order
    rr = scenes.random_rays(9, 5000)
    mrs, t2 = bvh.trace_diffuse(rr["org"], rr["dir"])
    rr["tmin"] = 0.0
    ref2 = O.brute_closest(small_scene, rr)
    assert mrs > 0
    assert np.array_equal(t2.view(np.uint32), np.where(ref2["prim"] >= 0, ref2["t"], np.float32(1e30)).view(np.uint32))
    # RGBA: sky where the oracle misses, shaded where it hits
    img = bvh.trace_rgba(64, 48, (0.0, 20.0, -90.0))
    assert img.shape == (64 * 48,) and np.all((img >> 24) == 255)


def test_exports_are_valid_bvhs(cuda, small_scene):
    bvh = lib.BVH(small_scene)
    ex = bvh.exports()
    n = small_scene.shape[0]
    pk = ex["packed"].reshape(-1, 12)
    assert pk.shape[0] == n
    assert sorted(pk[:, 9].astype(np.int64).tolist()) == list(range(n))
    assert np.array_equal(pk[:, :9], small_scene[pk[:, 9].astype(np.int64)])
    assert np.array_equal(ex["soa"].T, pk[:, :9])
    skips = ex["dfs"].reshape(-1, 8)[:, 7].view(np.int32)
    assert skips[0] == -1 and (skips == -2).sum() == 0
    assert np.array_equal(O.fix_skips(ex["dfs"]), ex["dfs"])
    rays = scenes.random_rays(21, 5000)
    assert_hits_equal(O.trace_closest_dfs(ex["dfs"], ex["packed"], rays), O.brute_closest(small_scene, rays), "dfs")
    # BVH4 export: every child box (fp16, rounded outward) holds its subtree
    b4 = ex["bvh4"].reshape(-1, 64)
    halfs = b4[:, :48].copy().view(np.float16).astype(np.float32).reshape(-1, 3, 8)
    child = b4[:, 48:].copy().view(np.int32)
    tri_lo = small_scene.reshape(-1, 3, 3).min(1)
    tri_hi = small_scene.reshape(-1, 3, 3).max(1)
    order = pk[:, 9].astype(np.int64)

    def subtree_box(c):
        if c <= -2:
            e = -(c + 2)
            ids = order[(e >> 3):(e >> 3) + (e & 7) + 1]
            return tri_lo[ids].min(0), tri_hi[ids].max(0)
        los, his = zip(*[subtree_box(k) for k in child[c] if k != -1])
        return np.min(los, 0), np.max(his, 0)

    for i in range(0, b4.shape[0], max(1, b4.shape[0] // 200)):
        for k in range(4):
            c = child[i, k]
            if c == -1:
                continue
            lo, hi = subtree_box(c)
            assert np.all(halfs[i, :, k] <= lo) and np.all(halfs[i, :, 4 + k] >= hi)
    assert ex["num_cwbvh"] == bvh.stats()["num_nodes"]


def _d2h(ptr, nbytes):
    """Device bytes to a host array (a synchronous copy, after all queued work)."""
    from cuda.bindings import runtime as cudart
    out = np.empty(nbytes, np.uint8)
    (err,) = cudart.cudaMemcpy(out.ctypes.data, ptr, nbytes, cudart.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == cudart.cudaError_t.cudaSuccess, err
    return out


def test_build_is_deterministic_and_sane(cuda):
    tris = scenes.scene_meshes(2, 120_000)
    a, b = lib.BVH(tris), lib.BVH(tris)
    sa = a.stats()
    assert sa["num_tris"] == tris.shape[0] and sa["bins"] == 32 and sa["max_leaf"] == 2
    assert 1 <= sa["depth"] <= 64
    la, lb = a.layout(), b.layout()
    assert la[1] == lb[1] and la[3] == lb[3] == tris.shape[0]
    assert np.array_equal(_d2h(la[0], la[1] * 80), _d2h(lb[0], lb[1] * 80))
    assert np.array_equal(_d2h(la[2], la[3] * 48), _d2h(lb[2], lb[3] * 48))
    assert sa["sah_cost"] > 0 and sa["build_ms"] > 0


def test_tlas_two_level_vs_oracle(cuda):
    rs = np.random.RandomState(5)
    blas_tris = [scenes.scene_meshes(10 + i, 3000 + 1000 * i, box=6.0, lo=200, hi=800, ground=False)
                 for i in range(4)]
    blases = [lib.BVH(t) for t in blas_tris]
    ninst = 24
    insts = (lib.RtInstance * ninst)()
    xf = []
    for k in range(ninst):
        R = scenes.rotations(rs.uniform(size=(1, 3)))[0] * rs.uniform(0.5, 2.0)
        t = rs.uniform(-40, 40, 3)
        M = np.concatenate([R, t[:, None]], 1).astype(np.float32)
        xf.append(M)
        insts[k].xform[:] = M.ravel().tolist()
        insts[k].blas = k % 4
    L = lib.load()
    import ctypes as C
    arr = (C.c_void_p * 4)(*[b.h for b in blases])
    tl = L.cudaTLAS_build(arr, 4, insts, ninst)
    assert tl, lib.last_error()
    try:
        inv = np.zeros((ninst, 12), np.float32)
        assert L.cudaTLAS_getInverseTransforms(tl, inv.ctypes.data, ninst) == 0
        # oracle side: restated builder per BLAS + LBVH over world boxes
        obs = [O.OracleBVH(t, 32, 4) for t in blas_tris]
        node_off = np.cumsum([0] + [o.dfs.size // 8 for o in obs]).astype(np.int32)
        tri_off = np.cumsum([0] + [o.packed.size // 12 for o in obs]).astype(np.int32)
        bdfs = np.concatenate([o.dfs for o in obs])
        bpk = np.concatenate([o.packed for o in obs])
        wb = []
        for k in range(ninst):
            v = blas_tris[k % 4].reshape(-1, 3).astype(np.float64) @ xf[k][:, :3].T.astype(np.float64) + xf[k][:, 3]
            lo, hi = v.min(0), v.max(0)
            pad = 1e-4 * (np.abs(v).max() + 1)
            wb.append(np.concatenate([lo - pad, hi + pad]))
        tnodes, tord = O.tlas_fast(np.array(wb, np.float32))
        tnodes = O.fix_skips(tnodes)
        # half the rays aimed at instance centres, half random
        rays = scenes.random_rays(33, 20000)
        tgt = np.array([m[:, 3] for m in xf])[rs.randint(0, ninst, 10000)] + rs.normal(0, 1.5, (10000, 3))
        d = tgt - rays["org"][:10000]
        rays["dir"][:10000] = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        hits = np.zeros(rays.shape[0], HIT_DTYPE)
        inst_ref = np.zeros(rays.shape[0], np.int32)
        iblas = np.array([k % 4 for k in range(ninst)], np.int32)
        Lo = O.lib()
        Lo.orc_trace_closest_two_level(tnodes.ctypes.data, tnodes.size // 8, tord.ctypes.data, inv.ctypes.data,
                                       iblas.ctypes.data, ninst, bdfs.ctypes.data, node_off.ctypes.data,
                                       bpk.ctypes.data, tri_off.ctypes.data, rays.ctypes.data, rays.shape[0],
                                       hits.ctypes.data, inst_ref.ctypes.data, 0)
        occ_ref = np.zeros(rays.shape[0], np.uint8)
        Lo.orc_trace_any_two_level(tnodes.ctypes.data, tnodes.size // 8, tord.ctypes.data, inv.ctypes.data,
                                   iblas.ctypes.data, ninst, bdfs.ctypes.data, node_off.ctypes.data,
                                   bpk.ctypes.data, tri_off.ctypes.data, rays.ctypes.data, rays.shape[0],
                                   occ_ref.ctypes.data, 0)
        import torch
        d_rays = _dev(torch, rays)
        d_hits = torch.empty(rays.shape[0] * 16, dtype=torch.uint8, device="cuda")
        d_inst = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
        d_occ = torch.empty(rays.shape[0], dtype=torch.uint8, device="cuda")
        assert L.cudaTLAS_traceClosest(tl, d_rays.data_ptr(), rays.shape[0], d_hits.data_ptr(), d_inst.data_ptr(),
                                       None) == 0
        assert L.cudaTLAS_traceAny(tl, d_rays.data_ptr(), rays.shape[0], d_occ.data_ptr(), None) == 0
        torch.cuda.synchronize()
        got = d_hits.cpu().numpy().view(HIT_DTYPE)
        assert_hits_equal(got, hits, "tlas")
        assert np.array_equal(d_inst.cpu().numpy(), inst_ref)
        assert np.array_equal(d_occ.cpu().numpy(), occ_ref)
        assert (hits["prim"] >= 0).mean() > 0.05
    finally:
        L.cudaTLAS_destroy(tl)


def _oracle_two_level(blas_tris, xf, bidx, inv, rays):
    """The oracle's two-level walk (restated builder per BLAS, LBVH over
    padded world boxes): closest hits, instance ids and occlusion flags."""
    obs = [O.OracleBVH(t, 32, 4) for t in blas_tris]
    node_off = np.cumsum([0] + [o.dfs.size // 8 for o in obs]).astype(np.int32)
    tri_off = np.cumsum([0] + [o.packed.size // 12 for o in obs]).astype(np.int32)
    bdfs = np.concatenate([o.dfs for o in obs])
    bpk = np.concatenate([o.packed for o in obs])
    ninst = len(bidx)
    wb = []
    for k in range(ninst):
        v = blas_tris[bidx[k]].reshape(-1, 3).astype(np.float64) @ xf[k][:, :3].T.astype(np.float64) + xf[k][:, 3]
        pad = 1e-4 * (np.abs(v).max() + 1)
        wb.append(np.concatenate([v.min(0) - pad, v.max(0) + pad]))
    tnodes, tord = O.tlas_fast(np.array(wb, np.float32))
    tnodes = O.fix_skips(tnodes)
    iblas = np.ascontiguousarray(bidx, np.int32)
    inv = np.ascontiguousarray(inv, np.float32)
    hits = np.zeros(rays.shape[0], HIT_DTYPE)
    inst_ref = np.zeros(rays.shape[0], np.int32)
    occ_ref = np.zeros(rays.shape[0], np.uint8)
    Lo = O.lib()
    args = (tnodes.ctypes.data, tnodes.size // 8, tord.ctypes.data, inv.ctypes.data, iblas.ctypes.data, ninst,
            bdfs.ctypes.data, node_off.ctypes.data, bpk.ctypes.data, tri_off.ctypes.data, rays.ctypes.data,
            rays.shape[0])
    Lo.orc_trace_closest_two_level(*args, hits.ctypes.data, inst_ref.ctypes.data, 0)
    Lo.orc_trace_any_two_level(*args, occ_ref.ctypes.data, 0)
    return hits, inst_ref, occ_ref


def test_tlas_rotated_floored_instances_vs_oracle(cuda):
    """Two-level traversal on the path tracer's kind of scene -- BLASes of
    mesh clusters over a two-triangle floor, rotated and scaled instances
    whose boxes overlap -- against the oracle's two-level walk: camera
    rays, bounce rays from their hits, and rays grazing the instances'
    floor planes and box faces, where any culling that is not conservative
    (the instance world boxes, the object-space box tested after entering
    an instance) shows up as a changed hit."""
    import torch
    blas_tris, xf, bidx, _, _ = scenes.instanced_scene(3, 240_000, nblas=8, ninst=48, world=100.0)
    tl = lib.TLAS([lib.BVH(t) for t in blas_tris], xf, bidx)
    try:
        rng = np.random.default_rng(4)
        cam = scenes.pinhole_rays(480, 270, scenes.PT_CAM_EYE, scenes.PT_CAM_TARGET, vfov_deg=50.0)
        parts = [cam]
        d_cam = _dev(torch, cam)
        d_h = torch.empty(cam.shape[0] * 16, dtype=torch.uint8, device="cuda")
        tl.closest(d_cam, cam.shape[0], d_h)
        torch.cuda.synchronize()
        h = d_h.cpu().numpy().view(HIT_DTYPE)
        hit = h["prim"] >= 0
        # bounce rays: uniform directions on the side of the incoming ray
        o = cam["org"][hit] + cam["dir"][hit] * h["t"][hit][:, None]
        dn = rng.normal(size=(int(hit.sum()), 3)).astype(np.float32)
        dn /= np.linalg.norm(dn, axis=1, keepdims=True)
        dn = np.where((dn * cam["dir"][hit]).sum(1, keepdims=True) > 0, -dn, dn)
        bnc = np.zeros(dn.shape[0], RAY_DTYPE)
        bnc["org"], bnc["dir"], bnc["tmin"], bnc["tmax"] = o + dn * np.float32(1e-3), dn, 1e-3, 1e30
        parts.append(bnc)
        # grazing rays: in each instance's floor plane (and the planes of its
        # object box faces), aimed across the instance with a tiny tilt
        for k in range(len(bidx)):
            v = blas_tris[bidx[k]].reshape(-1, 3).astype(np.float64)
            lo, hi = v.min(0), v.max(0)
            M = xf[k].astype(np.float64)
            m = 400
            q = rng.uniform(lo, hi, (m, 3))
            ax = rng.integers(0, 3, m)
            face = np.where(rng.random(m) < 0.5, lo[ax], hi[ax])
            q[np.arange(m), ax] = face
            q[: m // 4, 1] = v[:6, 1].min()  # the floor's plane
            dl = rng.normal(size=(m, 3))
            dl[np.arange(m), ax] *= 1e-4
            dl[: m // 4, 1] *= 1e-4
            dl /= np.linalg.norm(dl, axis=1, keepdims=True)
            wq, wd = q @ M[:, :3].T + M[:, 3], dl @ M[:, :3].T
            wd /= np.linalg.norm(wd, axis=1, keepdims=True)
            g = np.zeros(m, RAY_DTYPE)
            g["org"], g["dir"], g["tmin"], g["tmax"] = wq - wd * 50.0, wd, 0.0, 1e30
            parts.append(g)
        rays = np.ascontiguousarray(np.concatenate(parts))
        ref, inst_ref, occ_ref = _oracle_two_level(blas_tris, xf, bidx, tl.inverse(), rays)
        n = rays.shape[0]
        d_rays = _dev(torch, rays)
        d_hits = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
        d_inst = torch.empty(n, dtype=torch.int32, device="cuda")
        d_occ = torch.empty(n, dtype=torch.uint8, device="cuda")
        tl.closest(d_rays, n, d_hits, d_inst)
        tl.any(d_rays, n, d_occ)
        torch.cuda.synchronize()
        assert_hits_equal(d_hits.cpu().numpy().view(HIT_DTYPE), ref, "floored instances")
        assert np.array_equal(d_inst.cpu().numpy(), inst_ref)
        assert np.array_equal(d_occ.cpu().numpy(), occ_ref)
        assert (ref["prim"] >= 0).mean() > 0.3
    finally:
        tl.close()


def test_tlas_set_transforms_equals_a_fresh_build(cuda):
    """cudaTLAS_setTransforms moves every instance and changes BLAS choices in
    place: traces afterwards are byte-identical to those of a TLAS built with
    the new instances, and a path tracer created before the move renders
    exactly what one created on the new TLAS renders (it reloads transforms
    and light areas at its next render)."""
    import torch
    rs = np.random.RandomState(8)
    blases = [lib.BVH(scenes.scene_meshes(20 + i, 2000, box=30.0, lo=200, hi=800, ground=False)) for i in range(3)]
    n = 16

    def instances(seed):
        r = np.random.RandomState(seed)
        xf = [np.concatenate([scenes.rotations(r.uniform(size=(1, 3)))[0] * r.uniform(0.5, 2.0),
                              r.uniform(-30, 30, 3)[:, None]], 1).astype(np.float32) for _ in range(n)]
        return np.array(xf), r.randint(0, 3, n)

    xa, ba = instances(1)
    xb, bb = instances(2)
    alb = np.full((n, 3), 0.6, np.float32)
    emi = np.zeros((n, 3), np.float32)
    emi[[0, 5]] = 5.0
    cam = lib.make_camera((0.0, 0.0, -90.0), (0.0, 0.0, 0.0))
    W, H = 128, 72
    img = [torch.zeros(W * H * 3, dtype=torch.float32, device="cuda") for _ in range(3)]
    moved = lib.TLAS(blases, xa, ba)
    pt = lib.PathTracer(moved, alb, emi)
    pt.render(cam, W, H, 2, d_rgb=img[0])
    moved.set_transforms(xb, bb)
    fresh = lib.TLAS(blases, xb, bb)
    pt_fresh = lib.PathTracer(fresh, alb, emi)
    try:
        assert np.array_equal(moved.inverse(), fresh.inverse())
        rays = scenes.random_rays(61, 20000)
        d = xb[rs.randint(0, n, rays.shape[0]), :, 3] + rs.normal(0, 1.0, (rays.shape[0], 3)) - rays["org"]
        rays["dir"] = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        d_rays = _dev(torch, rays)
        out = []
        for tl in (moved, fresh):
            d_hits = torch.empty(rays.shape[0] * 16, dtype=torch.uint8, device="cuda")
            d_inst = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
            d_occ = torch.empty(rays.shape[0], dtype=torch.uint8, device="cuda")
            tl.closest(d_rays, rays.shape[0], d_hits, d_inst)
            tl.any(d_rays, rays.shape[0], d_occ)
            torch.cuda.synchronize()
            out.append((d_hits.cpu().numpy(), d_inst.cpu().numpy(), d_occ.cpu().numpy()))
        for a, b in zip(*out):
            assert np.array_equal(a, b)
        assert (out[0][1] >= 0).mean() > 0.05
        pt.render(cam, W, H, 2, d_rgb=img[1])
        pt_fresh.render(cam, W, H, 2, d_rgb=img[2])
        torch.cuda.synchronize()
        a, b, f = (x.cpu().numpy() for x in img)
        assert np.array_equal(b.view(np.uint32), f.view(np.uint32))
        assert b.sum() > 0 and not np.array_equal(a, b)
        assert pt.stats()["light_tris"] == pt_fresh.stats()["light_tris"]
    finally:
        pt_fresh.close()
        pt.close()
        fresh.close()
        moved.close()


def test_host_traces_over_replicas_equal_one_handle(cuda):
    """cudaBVH_traceClosestHostMulti / AnyHostMulti: a host batch split over
    replicas (here several handles on the one GPU of this box, each with its
    own host thread and pipeline) gives the single handle's results byte for
    byte, for batches longer and shorter than the replica count; bad
    arguments are rejected."""
    import ctypes as C
    tris = scenes.scene_meshes(31, 30_000, box=30.0, lo=300, hi=3000)
    rays = scenes.scene_rays(tris, 60_001, seed=9)
    reps = [lib.BVH(tris) for _ in range(3)]
    try:
        want = reps[0].closest_host(rays)
        want_occ = reps[0].any_host(rays)
        assert (want["prim"] >= 0).mean() > 0.2
        for k in (1, 2, 3):
            got = lib.trace_host_multi(reps[:k], rays)
            assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), f"{k} replicas"
            assert np.array_equal(lib.trace_host_multi(reps[:k], rays, any_hit=True), want_occ)
        few = np.ascontiguousarray(rays[:2])
        assert np.array_equal(lib.trace_host_multi(reps, few).view(np.uint8), want[:2].view(np.uint8))
        assert lib.trace_host_multi(reps, rays[:0]).shape == (0,)
        L = lib.load()
        hs = (C.c_void_p * 2)(reps[0].h, None)
        out = np.zeros(4, HIT_DTYPE)
        assert L.cudaBVH_traceClosestHostMulti(hs, 2, few.ctypes.data, 2, out.ctypes.data) == -1  # RT_ERR_INVALID
        assert L.cudaBVH_traceClosestHostMulti(hs, 0, few.ctypes.data, 2, out.ctypes.data) == -1  # RT_ERR_INVALID
    finally:
        for b in reps:
            b.close()


def test_counters_match_closest_results(cuda, small_scene):
    import torch
    bvh = lib.BVH(small_scene)
    rays = scenes.random_rays(44, 10000)
    d_rays = _dev(torch, rays)
    d_cnt = torch.zeros(rays.shape[0] * 2, dtype=torch.int32, device="cuda")
    bvh.counters(d_rays, rays.shape[0], d_cnt)
    torch.cuda.synchronize()
    c = d_cnt.cpu().numpy().reshape(-1, 2)
    assert c[:, 0].min() >= 1 and c[:, 1].mean() > 0


@pytest.mark.parametrize("any_hit", [False, True])
def test_work_counts_equal_the_oracle_walk(cuda, any_hit):
    """The kernel's per-ray node visits and triangle tests (the counts bench.py
    turns into algorithmic bytes) equal the oracle's restated 8-wide walk at
    the kernel's walk shape (node visits per round, pending triangle sets),
    ray for ray, on the library's own nodes, for incoherent diffuse rays."""
    import torch
    tris = scenes.scene_meshes(13, 20000, box=30.0, lo=200, hi=2000)
    bvh = lib.BVH(tris)
    try:
        rays = scenes.scene_rays(tris, 8192, seed=8)[4096:]
        pn, n_nodes, pt, n_recs = bvh.layout()
        nodes = _d2h(pn, n_nodes * 80).view(np.uint32).reshape(n_nodes, 20)
        recs = _d2h(pt, n_recs * 48).view(np.float32).reshape(n_recs, 12)
        n = rays.shape[0]
        d_rays = _dev(torch, rays)
        d_cnt = torch.zeros(n * 2, dtype=torch.int32, device="cuda")
        bvh.counters(d_rays, n, d_cnt, any_hit=any_hit)
        torch.cuda.synchronize()
        got = d_cnt.cpu().numpy().view(np.uint32).reshape(n, 2)
        out, ref = O.walk_bvh8(nodes, recs, rays, any_hit=any_hit)
        assert np.array_equal(got, ref), f"{int((got != ref).any(1).sum())} of {n} rays differ"
        if any_hit:
            assert np.array_equal(gpu_any(bvh, rays), out)
        else:
            assert_hits_equal(gpu_closest(bvh, rays), out, "8-wide walk")
        assert got[:, 0].mean() > 4 and got[:, 1].mean() > 2  # deep, incoherent walks
    finally:
        bvh.close()


def test_path_tracer_vs_fp64_oracle(cuda):
    """Wavefront path tracer (the 1080p TLAS workload, reduced size) against the FP64
    oracle on every pixel: the same paths (identical extension and shadow ray
    counts) and radiance within 1e-4 mean relative error."""
    import torch
    blases, xf, bidx, alb, emi = scenes.instanced_scene(2, 120_000, nblas=4, ninst=24, world=30.0, emissive_frac=0.25)
    bvhs = [lib.BVH(t) for t in blases]
    tl = lib.TLAS(bvhs, xf, bidx)
    pt = lib.PathTracer(tl, alb, emi)
    W, H, spp = 96, 64, 4
    cam = lib.make_camera((0.0, 8.0, -45.0), (0.0, 0.0, 0.0), vfov=60.0)
    d_rgb = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    pt.render(cam, W, H, spp, 4, 2, 7, d_rgb)
    torch.cuda.synchronize()
    img = d_rgb.cpu().numpy().reshape(-1, 3).astype(np.float64)
    st = pt.stats()
    orc = O.OraclePT(blases, xf, bidx, tl.inverse(), alb, emi)
    ref, counts = orc.pixels(lib.camera_basis(cam, W, H), W, H, spp, np.arange(W * H), 4, 2, 7)
    assert st["extension_rays"] == counts[0] and st["shadow_rays"] == counts[1]
    assert ref.sum() > 0 and (ref.max(1) > 0).mean() > 0.3
    mre = np.abs(img - ref).sum() / np.abs(ref).sum()
    assert mre < 1e-4, mre
    # rendering twice gives the same image (deterministic accumulation)
    d2 = torch.zeros_like(d_rgb)
    pt.render(cam, W, H, spp, 4, 2, 7, d2)
    torch.cuda.synchronize()
    assert torch.equal(d_rgb, d2)


@pytest.mark.parametrize("groups", ["1", "3"])
def test_batched_graph_build_equals_host_loop_build(cuda, monkeypatch, groups):
    """rtBatch_build's one-graph build (level loops as conditional WHILE
    nodes, counts kept on the device) writes the same 8-wide nodes and
    triangle records, byte for byte, as the host-driven level loop, on
    scenes of 1 to 60,000 triangles (leaf roots, small-task roots and deep
    large-task levels); also when both build the scenes in three groups and
    merge them into one layout (structure checked in the build)."""
    monkeypatch.setenv("RTB200_BATCH_GROUPS", groups)
    monkeypatch.setenv("RTB200_VALIDATE", "1")
    sizes = [1, 2, 3, 700, 1024, 1025, 60000, 5000, 30000, 9]
    tris = [scenes.scene_meshes(300 + i, n, box=30.0, lo=min(n, 100), hi=max(min(n, 4000), 100), ground=False)
            if n > 3 else np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]] * n, np.float32) + np.float32(i)
            for i, n in enumerate(sizes)]
    out = []
    for host_loop in (False, True):
        b = lib.Batch(tris, host_loop=host_loop)
        try:
            pn, n_nodes, pt, n_recs = b.layout()
            out.append((_d2h(pn, n_nodes * 80), _d2h(pt, n_recs * 48)))
        finally:
            b.close()
    (ga, gb), (ha, hb) = out
    assert ga.size == ha.size and gb.size == hb.size and gb.size == sum(sizes) * 48
    assert np.array_equal(ga, ha), "8-wide nodes differ"
    assert np.array_equal(gb, hb), "triangle records differ"


@pytest.mark.parametrize("groups", ["1", "4"])
def test_batched_scenes_equal_per_scene_calls(cuda, monkeypatch, groups):
    """rtBatch_*: one multi-scene build and one persistent launch (plain and
    replayed from a CUDA graph) give exactly the per-scene results,
    including a 1-triangle scene and scenes without rays; the same when the
    scenes are built in four groups and merged."""
    import torch
    monkeypatch.setenv("RTB200_BATCH_GROUPS", groups)
    sizes = [1, 3, 250, 5000, 20000, 777, 40000, 12]
    tris = [scenes.scene_meshes(100 + i, n, box=30.0, lo=min(n, 100), hi=max(min(n, 2000), 100), ground=False)
            if n > 2 else np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]] * n, np.float32) + np.float32(i)
            for i, n in enumerate(sizes)]
    nr = [3000, 0, 2000, 8000, 10000, 0, 12000, 500]
    rays = [scenes.random_rays(200 + i, k, box=40.0) for i, k in enumerate(nr)]
    off = np.concatenate([[0], np.cumsum(nr)]).astype(np.int32)
    allr = np.concatenate(rays)
    b = lib.Batch(tris)
    d_rays = _dev(torch, allr)
    d_off = torch.from_numpy(off).cuda()
    n = allr.shape[0]
    d_h = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    d_g = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    d_o = torch.empty(n, dtype=torch.uint8, device="cuda")
    b.closest(d_rays, d_off, n, d_h)
    b.graph(d_rays, d_off, n, d_g)
    b.graph(d_rays, d_off, n, d_g)  # replay
    b.any(d_rays, d_off, n, d_o)
    torch.cuda.synchronize()
    got = d_h.cpu().numpy().view(HIT_DTYPE)
    assert np.array_equal(d_g.cpu().numpy(), d_h.cpu().numpy())
    occ = d_o.cpu().numpy()
    for i, t in enumerate(tris):
        if nr[i] == 0:
            continue
        ref = O.brute_closest(t, rays[i])
        assert_hits_equal(got[off[i]:off[i + 1]], ref, f"scene {i}")
        assert np.array_equal(occ[off[i]:off[i + 1]], O.brute_any(t, rays[i]))
    ctas, iters = b.autotune(d_rays, d_off, n, d_h)
    t = b.tuning()
    assert 1 <= ctas <= 8 and iters in (2, 3, 4) and t["node_iters"] == iters
    assert t["block"] in (64, 128, 256) and t["shared_stack"] in (4, 8, 12) and 8 <= t["warps_per_sm"] <= 32
    b.graph(d_rays, d_off, n, d_g)
    torch.cuda.synchronize()
    assert np.array_equal(d_g.cpu().numpy(), d_h.cpu().numpy())
    # every launch shape the tuner can pick gives the same records
    for shape in ((8, 2, 64, 8), (32, 4, 256, 8), (16, 3, 128, 8), (24, 4, 128, 4), (32, 2, 128, 12)):
        b.set_tuning_ex(*shape)
        d_x = torch.empty_like(d_h)
        b.closest(d_rays, d_off, n, d_x)
        d_y = torch.empty_like(d_g)
        b.graph(d_rays, d_off, n, d_y)
        torch.cuda.synchronize()
        assert torch.equal(d_x, d_h) and torch.equal(d_y, d_h), shape


def test_grouped_batch_build_pinned_and_pageable(cuda, monkeypatch):
    """A batch built in two scene groups whose builds overlap the upload:
    from page-locked input (every group's copy queued at once) and from
    pageable input (each copy issued after the previous group's build was
    launched) the layout is the same byte for byte, and its closest and any
    hits equal those of one build over all scenes on every ray."""
    import torch
    sizes = [40000, 3, 25000, 1, 60000, 800, 15000, 5000]
    tris = [scenes.scene_meshes(500 + i, k, box=30.0, lo=min(k, 100), hi=max(min(k, 4000), 100), ground=False)
            if k > 3 else np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]] * k, np.float32) + np.float32(i)
            for i, k in enumerate(sizes)]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    pageable = np.concatenate(tris)
    pin = torch.empty(pageable.nbytes, dtype=torch.uint8, pin_memory=True)
    pinned = pin.numpy().view(np.float32).reshape(-1, 9)
    pinned[:] = pageable
    nr = [4000, 500, 3000, 100, 6000, 1000, 2000, 1500]
    rays = np.concatenate([scenes.random_rays(600 + i, k, box=40.0) for i, k in enumerate(nr)])
    roff = np.concatenate([[0], np.cumsum(nr)]).astype(np.int32)
    d_rays, d_off, n = _dev(torch, rays), torch.from_numpy(roff).cuda(), rays.shape[0]
    monkeypatch.setenv("RTB200_VALIDATE", "1")
    layouts, hits, occ = [], [], []
    for groups, src in (("2", pinned), ("2", pageable), ("1", pageable)):
        monkeypatch.setenv("RTB200_BATCH_GROUPS", groups)
        b = lib.Batch(all_tris=src, tri_offsets=off)
        try:
            pn, n_nodes, pt, n_recs = b.layout()
            layouts.append((_d2h(pn, n_nodes * 80), _d2h(pt, n_recs * 48)))
            d_h = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
            d_o = torch.empty(n, dtype=torch.uint8, device="cuda")
            b.closest(d_rays, d_off, n, d_h)
            b.any(d_rays, d_off, n, d_o)
            torch.cuda.synchronize()
            hits.append(d_h.cpu().numpy())
            occ.append(d_o.cpu().numpy())
        finally:
            b.close()
    assert np.array_equal(layouts[0][0], layouts[1][0]) and np.array_equal(layouts[0][1], layouts[1][1])
    assert layouts[0][0].size == layouts[2][0].size  # the same nodes, in another order
    assert (hits[0].view(HIT_DTYPE)["prim"] >= 0).mean() > 0.05
    assert np.array_equal(hits[0], hits[2]) and np.array_equal(occ[0], occ[2])


def test_pipelined_host_calls_equal_device_calls(cuda):
    """Host-buffer calls larger than one 512K-ray piece run as a pipeline of
    pieces (copy in, trace on two alternating streams, copy out): results
    equal the device-buffer path's, for pinned and pageable host memory,
    closest and any hit, with a ragged last piece."""
    import torch
    tris = scenes.scene_meshes(61, 100_000, box=40.0)
    bvh = lib.BVH(tris)
    rays = scenes.random_rays(62, 1_200_001, box=50.0)
    n = rays.shape[0]
    d_rays = _dev(torch, rays)
    d_h = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    d_o = torch.empty(n, dtype=torch.uint8, device="cuda")
    bvh.closest(d_rays, n, d_h)
    bvh.any(d_rays, n, d_o)
    torch.cuda.synchronize()
    ref_h, ref_o = d_h.cpu().numpy(), d_o.cpu().numpy()
    L = lib.load()
    p_r = torch.empty(n * 32, dtype=torch.uint8, pin_memory=True)
    p_r.numpy()[:] = rays.view(np.uint8).reshape(-1)
    p_h = torch.zeros(n * 16, dtype=torch.uint8, pin_memory=True)
    p_o = torch.zeros(n, dtype=torch.uint8, pin_memory=True)
    for _ in range(2):  # repeated calls reuse the staging buffers and events
        assert L.cudaBVH_traceClosestHost(bvh.h, p_r.data_ptr(), n, p_h.data_ptr()) == 0, lib.last_error()
        assert L.cudaBVH_traceAnyHost(bvh.h, p_r.data_ptr(), n, p_o.data_ptr()) == 0, lib.last_error()
        assert np.array_equal(p_h.numpy(), ref_h) and np.array_equal(p_o.numpy(), ref_o)
    assert np.array_equal(bvh.closest_host(rays).view(np.uint8).reshape(-1), ref_h)  # pageable
    assert np.array_equal(bvh.any_host(rays), ref_o)
    assert 0.05 < (ref_h.view(HIT_DTYPE)["prim"] >= 0).mean() < 0.95
