"""BLAS from the application's vertex/index buffers, refit, and BVH blobs.

Every path must give the same hits, bit for bit, as a BLAS built with
cudaBVH_build from the equivalent host triangle soup (results are defined by
the triangle test and the tie rule alone, so equal triangles mean equal hits).
"""
import numpy as np
import pytest

from oracle import oracle as O
from rtb200 import lib, scenes
from rtb200.scenes import HIT_DTYPE

pytestmark = pytest.mark.gpu


def _dev(torch, arr):
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1).copy()).cuda()


def _hits(bvh, d_rays, n):
    import torch
    d_h = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    d_o = torch.empty(n, dtype=torch.uint8, device="cuda")
    bvh.closest(d_rays, n, d_h)
    bvh.any(d_rays, n, d_o)
    torch.cuda.synchronize()
    return d_h.cpu().numpy(), d_o.cpu().numpy()


def _indexed(tris):
    """Unique vertices and the index buffer that rebuilds `tris`."""
    v = tris.reshape(-1, 3)
    uniq, inv = np.unique(v, axis=0, return_inverse=True)
    return np.ascontiguousarray(uniq, np.float32), inv.reshape(-1).astype(np.uint32)


def _xform_rows(v, m):
    """((m0 x + m1 y) + m2 z) + m3 per row, every step rounded in fp32."""
    m = np.asarray(m, np.float32).reshape(3, 4)
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    out = np.empty_like(v)
    for r in range(3):
        out[:, r] = ((m[r, 0] * x + m[r, 1] * y) + m[r, 2] * z) + m[r, 3]
    return out


@pytest.fixture(scope="module")
def meshes():
    a = scenes.scene_meshes(41, 6000, box=30.0, lo=500, hi=2000, ground=False)
    b = scenes.scene_meshes(42, 3000, box=30.0, lo=500, hi=2000, ground=False)
    c = scenes.scene_meshes(43, 4000, box=30.0, lo=500, hi=2000, ground=False)
    rays = scenes.random_rays(44, 30000, box=40.0)
    return a, b, c, rays


def test_build_from_vertex_and_index_buffers(cuda, meshes):
    import torch
    a, b, c, rays = meshes
    # geometry 0: float3 vertices with a 16-byte stride, uint32 indices
    va, ia = _indexed(a)
    va4 = np.zeros((va.shape[0], 4), np.float32)
    va4[:, :3] = va
    # geometry 1: float3, 12-byte stride, no indices
    vb = b.reshape(-1, 3).astype(np.float32)
    # geometry 2: half3 (8-byte stride: xyz + pad), uint16 indices, 3x4 transform
    vc, ic = _indexed(c)
    assert vc.shape[0] < 65536
    vc16 = np.zeros((vc.shape[0], 4), np.float16)
    vc16[:, :3] = vc.astype(np.float16)
    m = np.array([0.8, -0.6, 0.0, 5.0, 0.6, 0.8, 0.0, -3.0, 0.0, 0.0, 1.0, 2.5], np.float32)
    d = [_dev(torch, va4), _dev(torch, ia), _dev(torch, vb), _dev(torch, vc16), _dev(torch, ic.astype(np.uint16))]
    G = lib.RtGeometry
    geoms = [G(d[0].data_ptr(), 16, lib.RT_VERTEX_FLOAT3, va.shape[0] - 1, d[1].data_ptr(), lib.RT_INDEX_UINT32,
               a.shape[0], None),
             G(d[2].data_ptr(), 12, lib.RT_VERTEX_FLOAT3, vb.shape[0] - 1, None, lib.RT_INDEX_NONE, b.shape[0], None),
             G(d[3].data_ptr(), 8, lib.RT_VERTEX_HALF3, vc.shape[0] - 1, d[4].data_ptr(), lib.RT_INDEX_UINT16,
               c.shape[0], m.ctypes.data)]
    torch.cuda.synchronize()
    got = lib.BVH.from_geometries(geoms)
    c_soup = _xform_rows(vc16[:, :3].astype(np.float32)[ic], m).reshape(-1, 9)
    soup = np.concatenate([va[ia].reshape(-1, 9), b, c_soup]).astype(np.float32)
    ref = lib.BVH(soup)
    d_rays = _dev(torch, rays)
    gh, go = _hits(got, d_rays, rays.shape[0])
    rh, ro = _hits(ref, d_rays, rays.shape[0])
    assert np.array_equal(gh, rh) and np.array_equal(go, ro)
    hits = gh.view(HIT_DTYPE)
    assert (hits["prim"] >= a.shape[0] + b.shape[0]).any()  # the transformed half geometry is hit too
    assert 0.05 < (hits["prim"] >= 0).mean() < 0.95


def test_geometry_errors_are_reported(cuda, meshes):
    import torch
    a = meshes[0]
    va, ia = _indexed(a)
    dv, di = _dev(torch, va), _dev(torch, ia)
    G = lib.RtGeometry
    with pytest.raises(lib.RtError):  # indices reach past max_vertex: refused, nothing read there
        lib.BVH.from_geometries([G(dv.data_ptr(), 12, lib.RT_VERTEX_FLOAT3, va.shape[0] // 2, di.data_ptr(),
                                   lib.RT_INDEX_UINT32, a.shape[0], None)])
    with pytest.raises(lib.RtError):  # misaligned vertex buffer
        lib.BVH.from_geometries([G(dv.data_ptr() + 2, 12, lib.RT_VERTEX_FLOAT3, va.shape[0] - 1, di.data_ptr(),
                                   lib.RT_INDEX_UINT32, a.shape[0], None)])
    with pytest.raises(lib.RtError):  # stride smaller than a vertex
        lib.BVH.from_geometries([G(dv.data_ptr(), 8, lib.RT_VERTEX_FLOAT3, va.shape[0] - 1, di.data_ptr(),
                                   lib.RT_INDEX_UINT32, a.shape[0], None)])
    with pytest.raises(lib.RtError):  # non-indexed triangles beyond max_vertex
        lib.BVH.from_geometries([G(dv.data_ptr(), 12, lib.RT_VERTEX_FLOAT3, 10, None, lib.RT_INDEX_NONE,
                                   a.shape[0], None)])


def test_refit_after_vertex_motion(cuda, meshes):
    import torch
    a, b, c, rays = meshes
    bvh = lib.BVH(a)
    # smooth deformation plus a translation: same triangles, new positions
    v = a.reshape(-1, 3).astype(np.float64)
    moved = (v + np.stack([np.sin(v[:, 1] * 0.2), 0.5 * np.cos(v[:, 0] * 0.1), np.full(len(v), 3.0)], 1))
    moved = moved.astype(np.float32).reshape(-1, 9)
    d_rays = _dev(torch, rays)
    bvh.refit(_dev(torch, moved))
    gh, go = _hits(bvh, d_rays, rays.shape[0])
    rh, ro = _hits(lib.BVH(moved), d_rays, rays.shape[0])
    assert np.array_equal(gh, rh) and np.array_equal(go, ro)
    assert np.array_equal(gh.view(HIT_DTYPE)["prim"], O.brute_closest(moved, rays)["prim"])
    bvh.validate()
    # refit back from vertex buffers
    vb = a.reshape(-1, 3).astype(np.float32)
    dvb = _dev(torch, vb)
    bvh.refit_geometries([lib.RtGeometry(dvb.data_ptr(), 12, lib.RT_VERTEX_FLOAT3, vb.shape[0] - 1, None,
                                         lib.RT_INDEX_NONE, a.shape[0], None)])
    gh2, go2 = _hits(bvh, d_rays, rays.shape[0])
    rh2, ro2 = _hits(lib.BVH(a), d_rays, rays.shape[0])
    assert np.array_equal(gh2, rh2) and np.array_equal(go2, ro2)


def test_blob_round_trip_and_rejections(cuda, meshes):
    import torch
    a, b, c, rays = meshes
    bvh = lib.BVH(a)
    blob = bvh.serialize()
    again = lib.BVH.deserialize(blob)
    d_rays = _dev(torch, rays)
    gh, go = _hits(again, d_rays, rays.shape[0])
    rh, ro = _hits(bvh, d_rays, rays.shape[0])
    assert np.array_equal(gh, rh) and np.array_equal(go, ro)
    assert again.stats()["num_nodes"] == bvh.stats()["num_nodes"]
    # host exports come from the stored binary BVH
    ea, eb = again.exports(), bvh.exports()
    for k in eb:
        assert np.array_equal(np.asarray(ea[k]), np.asarray(eb[k])), k
    assert again.serialize() == blob
    bad = bytearray(blob)
    bad[len(bad) // 2] ^= 0x40
    with pytest.raises(lib.RtError):  # checksum
        lib.BVH.deserialize(bytes(bad))
    with pytest.raises(lib.RtError):  # truncated
        lib.BVH.deserialize(blob[: len(blob) - 100])
    with pytest.raises(lib.RtError):  # not a blob
        lib.BVH.deserialize(b"X" * len(blob))
    bad = bytearray(blob)
    bad[8] = 99  # version
    with pytest.raises(lib.RtError):
        lib.BVH.deserialize(bytes(bad))
