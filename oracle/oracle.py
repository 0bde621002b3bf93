"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It loads ``oracle/liboracle.so`` (the restatement, see
oracle.h) and, when present, the reference objects compiled from the
reference's own sources into ``oracle/_ref/``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

RAY_DTYPE = np.dtype([("org", "<f4", 3), ("tmin", "<f4"), ("dir", "<f4", 3), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("prim", "<i4"), ("u", "<f4"), ("v", "<f4")])

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"oracle library missing: {path} (run `make -C oracle`)")
        L = C.CDLL(str(path))
        vp, i32, f32p, u32p = C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_uint32)
        L.orc_build.restype = vp
        L.orc_build.argtypes = [vp, i32, i32, i32]
        L.orc_free.argtypes = [vp]
        for name in ("orc_num_bvh2", "orc_num_dfs", "orc_num_packed", "orc_num_bvh4"):
            getattr(L, name).restype = i32
            getattr(L, name).argtypes = [vp]
        L.orc_dfs.restype = u32p
        L.orc_dfs.argtypes = [vp]
        L.orc_packed.restype = f32p
        L.orc_packed.argtypes = [vp]
        L.orc_bvh4.restype = vp
        L.orc_bvh4.argtypes = [vp]
        L.orc_orig_idx.restype = C.POINTER(C.c_int)
        L.orc_orig_idx.argtypes = [vp]
        L.orc_bounds.argtypes = [vp, f32p, f32p, f32p, f32p]
        L.orc_tlas_fast.restype = i32
        L.orc_tlas_fast.argtypes = [vp, i32, C.POINTER(u32p), C.POINTER(C.POINTER(C.c_int))]
        L.orc_free_ptr.argtypes = [vp]
        L.orc_trace_closest_dfs.argtypes = [vp, i32, vp, vp, i32, vp, i32, vp]
        L.orc_trace_any_dfs.argtypes = [vp, i32, vp, vp, i32, vp, i32]
        L.orc_brute_closest.argtypes = [vp, i32, vp, i32, vp, i32]
        L.orc_brute_any.argtypes = [vp, i32, vp, i32, vp, i32]
        L.orc_trace_closest_two_level.argtypes = [vp, i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, i32, vp, vp, i32]
        L.orc_trace_any_two_level.argtypes = [vp, i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, i32, vp, i32]
        L.orc_philox4x32_10.argtypes = [vp, vp, vp]
        L.orc_fix_skips.restype = i32
        L.orc_fix_skips.argtypes = [vp, i32]
        L.orc_f2h_rn.restype = C.c_uint16
        L.orc_f2h_rn.argtypes = [C.c_float]
        L.orc_pt_pixels.argtypes = [vp, vp, vp, vp, i32, vp, i32, vp]
        L.orc_walk_bvh8.restype = i32
        L.orc_walk_bvh8.argtypes = [vp, i32, vp, i32, vp, i32, i32, i32, i32, vp, vp, vp, i32]
        f32 = C.c_float
        L.orc_generate_rays.restype = i32
        L.orc_generate_rays.argtypes = [vp, i32, vp, vp, i32, i32, i32, C.c_uint32, f32, f32, f32, vp, f32, vp, vp,
                                        i32]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


class OracleBVH:
    """Restated reference builder (binned SAH BVH2 -> DFS, packed tris, BVH4)."""

    def __init__(self, tris: np.ndarray, nbins: int = 32, max_leaf: int = 4):
        tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
        self.n = tris.shape[0]
        self._tris = tris
        L = lib()
        self.h = L.orc_build(_p(tris), self.n, nbins, max_leaf)
        if not self.h:
            raise ValueError("oracle build failed (empty input?)")
        nd = L.orc_num_dfs(self.h)
        # dfs_ref: byte-identical to the reference export (skip placeholders
        # included); dfs: the same nodes with correct skip pointers.
        self.dfs_ref = np.ctypeslib.as_array(L.orc_dfs(self.h), shape=(nd * 8,)).copy()
        self.dfs = fix_skips(self.dfs_ref)
        npk = L.orc_num_packed(self.h)
        self.packed = np.ctypeslib.as_array(L.orc_packed(self.h), shape=(npk * 4,)).copy()
        nb4 = L.orc_num_bvh4(self.h)
        self.bvh4 = np.frombuffer(C.string_at(L.orc_bvh4(self.h), nb4 * 64), dtype=np.uint8).copy()
        self.orig_idx = np.ctypeslib.as_array(L.orc_orig_idx(self.h), shape=(npk // 3,)).copy()
        self.num_bvh2 = L.orc_num_bvh2(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    def closest(self, rays: np.ndarray, nthreads: int = 0, stats: bool = False):
        return trace_closest_dfs(self.dfs, self.packed, rays, nthreads, stats)

    def any(self, rays: np.ndarray, nthreads: int = 0):
        return trace_any_dfs(self.dfs, self.packed, rays, nthreads)


def trace_closest_dfs(dfs, packed, rays, nthreads=0, stats=False):
    rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
    dfs = np.ascontiguousarray(dfs, dtype=np.uint32)
    packed = np.ascontiguousarray(packed, dtype=np.float32)
    hits = np.zeros(rays.shape[0], dtype=HIT_DTYPE)
    st = np.zeros((rays.shape[0], 2), dtype=np.uint64) if stats else None
    lib().orc_trace_closest_dfs(_p(dfs), dfs.size // 8, _p(packed), _p(rays), rays.shape[0], _p(hits),
                                nthreads, _p(st) if stats else None)
    return (hits, st) if stats else hits


# the release kernel's walk shape: node visits per round, pending triangle sets
KERNEL_NITERS, KERNEL_SETS = 4, 2


def walk_bvh8(nodes, recs, rays, any_hit=False, niters=KERNEL_NITERS, sets=KERNEL_SETS, nthreads=0):
    """The engine's 8-wide walk restated on the CPU (orc_walk_bvh8).  nodes:
    (N, 20) u32 as laid out on the device; recs: (M, 12) f32 triangle
    records; niters node visits per round and `sets` (1 or 2) pending
    triangle sets per ray (the kernel's RTB_NODE_ITERS / RTB_TWO_SETS).
    Returns (hits or occlusion flags, counts (n, 2) u32 of node visits and
    triangle tests per ray); raises if a walk leaves the arrays."""
    rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32).reshape(-1, 20)
    recs = np.ascontiguousarray(recs, dtype=np.float32).reshape(-1, 12)
    n = rays.shape[0]
    counts = np.zeros((n, 2), dtype=np.uint32)
    out = np.zeros(n, dtype=np.uint8) if any_hit else np.zeros(n, dtype=HIT_DTYPE)
    bad = lib().orc_walk_bvh8(_p(nodes), nodes.shape[0], _p(recs), recs.shape[0], _p(rays), n, int(any_hit),
                              niters, sets, None if any_hit else _p(out), _p(out) if any_hit else None,
                              _p(counts), nthreads)
    if bad < 0:
        raise ValueError("walk_bvh8: niters must be >= 1 and sets 1 or 2")
    if bad:
        raise ValueError(f"walk_bvh8: {bad} walks left the node or record arrays")
    return out, counts


def trace_any_dfs(dfs, packed, rays, nthreads=0):
    rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
    dfs = np.ascontiguousarray(dfs, dtype=np.uint32)
    packed = np.ascontiguousarray(packed, dtype=np.float32)
    occ = np.zeros(rays.shape[0], dtype=np.uint8)
    lib().orc_trace_any_dfs(_p(dfs), dfs.size // 8, _p(packed), _p(rays), rays.shape[0], _p(occ), nthreads)
    return occ


def brute_closest(tris, rays, nthreads=0):
    tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
    rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
    hits = np.zeros(rays.shape[0], dtype=HIT_DTYPE)
    lib().orc_brute_closest(_p(tris), tris.shape[0], _p(rays), rays.shape[0], _p(hits), nthreads)
    return hits


def brute_any(tris, rays, nthreads=0):
    tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
    rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
    occ = np.zeros(rays.shape[0], dtype=np.uint8)
    lib().orc_brute_any(_p(tris), tris.shape[0], _p(rays), rays.shape[0], _p(occ), nthreads)
    return occ


def tlas_fast(aabbs: np.ndarray):
    """Restated cudaBVH_buildTLASFast: (nodes u32[8*m], ordered i32[n])."""
    aabbs = np.ascontiguousarray(aabbs, dtype=np.float32).reshape(-1, 6)
    L = lib()
    pn = C.POINTER(C.c_uint32)()
    po = C.POINTER(C.c_int)()
    m = L.orc_tlas_fast(_p(aabbs), aabbs.shape[0], C.byref(pn), C.byref(po))
    if m <= 0:
        return np.zeros(0, np.uint32), np.zeros(0, np.int32)
    nodes = np.ctypeslib.as_array(pn, shape=(m * 8,)).copy()
    ordered = np.ctypeslib.as_array(po, shape=(aabbs.shape[0],)).copy()
    L.orc_free_ptr(C.cast(pn, C.c_void_p))
    L.orc_free_ptr(C.cast(po, C.c_void_p))
    return nodes, ordered


def fix_skips(dfs: np.ndarray) -> np.ndarray:
    """Copy of a stackless export with every skip pointer recomputed."""
    out = np.ascontiguousarray(dfs, dtype=np.uint32).copy()
    if lib().orc_fix_skips(_p(out), out.size // 8) < 0:
        raise ValueError("not a preorder binary tree")
    return out


def generate_rays(tris, rays, hits, kind, count=0, seed=3, eps=1e-3, tmin=1e-3, tmax=1e30,
                  light_center=(0.0, 80.0, 0.0), light_size=1.0, nthreads=0):
    """Restated cudaBVH_generateRays: (rays, src) of the next bounce from a
    closest-hit batch; kind 0 diffuse, 1 shadow."""
    tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
    rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
    hits = np.ascontiguousarray(hits, dtype=HIT_DTYPE)
    n = rays.shape[0]
    cap = count if count > 0 else n
    out = np.zeros(cap, dtype=RAY_DTYPE)
    src = np.zeros(cap, dtype=np.int32)
    lc = np.ascontiguousarray(light_center, dtype=np.float32)
    m = lib().orc_generate_rays(_p(tris), tris.shape[0], _p(rays), _p(hits), n, int(kind), int(count),
                                seed & 0xFFFFFFFF, eps, tmin, tmax, _p(lc), light_size, _p(out), _p(src), nthreads)
    return out[:m], src[:m]


def philox4x32_10(ctr, key):
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32)
    key = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(_p(ctr), _p(key), _p(out))
    return out


def f2h(x: float) -> int:
    return int(lib().orc_f2h_rn(x))


# --------------------------------------------------------------------------
# Reference objects compiled from the reference's sources (oracle/_ref).
# --------------------------------------------------------------------------
class RefBackend:
    """The reference's layer/cuda_bvh_backend.cu, compiled as shipped
    (BVH_LAYER_MODE=1): its CPU builder and exports, no GPU needed."""

    def __init__(self, name: str = "libref_backend.so"):
        path = REF_DIR / name
        if not path.exists():
            raise FileNotFoundError(str(path))
        L = C.CDLL(str(path))
        vp, i32 = C.c_void_p, C.c_int
        L.cudaBVH_build.restype = vp
        L.cudaBVH_build.argtypes = [vp, i32]
        L.cudaBVH_destroy.argtypes = [vp]
        L.cudaBVH_getStacklessBVH2.restype = i32
        L.cudaBVH_getStacklessBVH2.argtypes = [vp, C.POINTER(C.POINTER(C.c_uint32))]
        L.cudaBVH_getPackedTris.restype = i32
        L.cudaBVH_getPackedTris.argtypes = [vp, C.POINTER(C.POINTER(C.c_float))]
        L.cudaBVH_getNodeData.restype = vp
        L.cudaBVH_getNodeData.argtypes = [vp]
        L.cudaBVH_getNumBVH4Nodes.restype = i32
        L.cudaBVH_getNumBVH4Nodes.argtypes = [vp]
        L.cudaBVH_getNumTris.restype = i32
        L.cudaBVH_getNumTris.argtypes = [vp]
        L.cudaBVH_getBounds.argtypes = [vp] + [C.POINTER(C.c_float)] * 4
        L.cudaBVH_getTriData.argtypes = [vp, C.POINTER(C.c_void_p * 9)]
        L.cudaBVH_buildTLASFast.restype = i32
        L.cudaBVH_buildTLASFast.argtypes = [vp, i32, C.POINTER(C.POINTER(C.c_uint32)),
                                            C.POINTER(C.POINTER(C.c_int))]
        L.cudaBVH_buildFromAABBs.restype = vp
        L.cudaBVH_buildFromAABBs.argtypes = [vp, i32]
        self.L = L

    def build_exports(self, tris: np.ndarray):
        """Build with the reference builder; return its exports as arrays."""
        tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
        h = self.L.cudaBVH_build(_p(tris), tris.shape[0])
        return self._exports(h)

    def build_from_aabbs(self, aabbs: np.ndarray):
        aabbs = np.ascontiguousarray(aabbs, dtype=np.float32).reshape(-1, 6)
        h = self.L.cudaBVH_buildFromAABBs(_p(aabbs), aabbs.shape[0])
        return self._exports(h)

    def _exports(self, h):
        L = self.L
        try:
            pd = C.POINTER(C.c_uint32)()
            nd = L.cudaBVH_getStacklessBVH2(h, C.byref(pd))
            dfs = np.ctypeslib.as_array(pd, shape=(nd * 8,)).copy()
            pp = C.POINTER(C.c_float)()
            npk = L.cudaBVH_getPackedTris(h, C.byref(pp))
            packed = np.ctypeslib.as_array(pp, shape=(npk * 4,)).copy()
            nb4 = L.cudaBVH_getNumBVH4Nodes(h)
            bvh4 = np.frombuffer(C.string_at(L.cudaBVH_getNodeData(h), nb4 * 64), dtype=np.uint8).copy()
            ptrs = (C.c_void_p * 9)()
            L.cudaBVH_getTriData(h, C.byref(ptrs))
            ntri = L.cudaBVH_getNumTris(h)
            soa = np.stack([np.ctypeslib.as_array(C.cast(ptrs[i], C.POINTER(C.c_float)), shape=(ntri,)).copy()
                            for i in range(9)]) if ntri else np.zeros((9, 0), np.float32)
            f = [C.c_float() for _ in range(4)]
            L.cudaBVH_getBounds(h, *[C.byref(x) for x in f])
            bounds = np.array([x.value for x in f], np.float32)
            return {"dfs": dfs, "packed": packed, "bvh4": bvh4, "soa": soa, "bounds": bounds}
        finally:
            L.cudaBVH_destroy(h)

    def tlas_fast(self, aabbs: np.ndarray):
        aabbs = np.ascontiguousarray(aabbs, dtype=np.float32).reshape(-1, 6)
        pn = C.POINTER(C.c_uint32)()
        po = C.POINTER(C.c_int)()
        m = self.L.cudaBVH_buildTLASFast(_p(aabbs), aabbs.shape[0], C.byref(pn), C.byref(po))
        nodes = np.ctypeslib.as_array(pn, shape=(m * 8,)).copy()
        ordered = np.ctypeslib.as_array(po, shape=(aabbs.shape[0],)).copy()
        libc = C.CDLL("libc.so.6")
        libc.free(C.cast(pn, C.c_void_p))
        libc.free(C.cast(po, C.c_void_p))
        return nodes, ordered


def ref_available(name: str = "libref_backend.so") -> bool:
    return (REF_DIR / name).exists()


def default_threads() -> int:
    return os.cpu_count() or 1


# --------------------------------------------------------------------------
# FP64 path-tracing oracle over an instanced scene.
# --------------------------------------------------------------------------
class _PTScene(C.Structure):
    _fields_ = [("tlas", C.c_void_p), ("tlas_nodes", C.c_int), ("tlas_ordered", C.c_void_p),
                ("inv12", C.c_void_p), ("fwd12", C.c_void_p), ("inst_blas", C.c_void_p), ("ninst", C.c_int),
                ("blas_dfs", C.c_void_p), ("node_off", C.c_void_p), ("blas_packed", C.c_void_p),
                ("tri_off", C.c_void_p), ("blas_tris9", C.c_void_p), ("blas_tri_base", C.c_void_p),
                ("blas_tri_count", C.c_void_p), ("albedo3", C.c_void_p), ("emission3", C.c_void_p)]


class _PTParams(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("spp", C.c_int), ("max_bounces", C.c_int),
                ("rr_start", C.c_int), ("seed", C.c_uint32)]


class OraclePT:
    """Two-level oracle scene (restated builder per BLAS, LBVH over padded
    world boxes) plus the FP64 path tracer."""

    def __init__(self, blases, xforms, blas_index, inv12, albedo, emission):
        self.obs = [OracleBVH(t, 32, 4) for t in blases]
        self.node_off = np.cumsum([0] + [o.dfs.size // 8 for o in self.obs]).astype(np.int32)
        self.tri_off = np.cumsum([0] + [o.packed.size // 12 for o in self.obs]).astype(np.int32)
        self.bdfs = np.concatenate([o.dfs for o in self.obs])
        self.bpk = np.concatenate([o.packed for o in self.obs])
        self.tris9 = np.concatenate([np.asarray(t, np.float32).reshape(-1, 9) for t in blases])
        self.tri_base = np.cumsum([0] + [len(t) for t in blases])[:-1].astype(np.int32)
        self.tri_count = np.array([len(t) for t in blases], np.int32)
        self.xf = np.ascontiguousarray(np.asarray(xforms, np.float32).reshape(-1, 12))
        self.inv = np.ascontiguousarray(np.asarray(inv12, np.float32).reshape(-1, 12))
        self.iblas = np.ascontiguousarray(blas_index, np.int32)
        self.albedo = np.ascontiguousarray(albedo, np.float32)
        self.emission = np.ascontiguousarray(emission, np.float32)
        wb = []
        for k in range(len(self.iblas)):
            v = np.asarray(blases[self.iblas[k]], np.float64).reshape(-1, 3)
            M = self.xf[k].reshape(3, 4).astype(np.float64)
            w = v @ M[:, :3].T + M[:, 3]
            pad = 1e-4 * (np.abs(w).max() + 1)
            wb.append(np.concatenate([w.min(0) - pad, w.max(0) + pad]))
        tn, self.tord = tlas_fast(np.array(wb, np.float32))
        self.tnodes = fix_skips(tn)
        self.scene = _PTScene(self.tnodes.ctypes.data, self.tnodes.size // 8, self.tord.ctypes.data,
                              self.inv.ctypes.data, self.xf.ctypes.data, self.iblas.ctypes.data, len(self.iblas),
                              self.bdfs.ctypes.data, self.node_off.ctypes.data, self.bpk.ctypes.data,
                              self.tri_off.ctypes.data, self.tris9.ctypes.data, self.tri_base.ctypes.data,
                              self.tri_count.ctypes.data, self.albedo.ctypes.data, self.emission.ctypes.data)

    def pixels(self, cam14, w, h, spp, pixels, max_bounces=4, rr_start=2, seed=1, nthreads=0):
        cam14 = np.ascontiguousarray(cam14, np.float32)
        px = np.ascontiguousarray(pixels, np.int32)
        out = np.zeros((px.size, 3), np.float64)
        counts = np.zeros(2, np.uint64)
        p = _PTParams(w, h, spp, max_bounces, rr_start, seed)
        lib().orc_pt_pixels(C.byref(self.scene), cam14.ctypes.data, C.byref(p), px.ctypes.data, px.size,
                            out.ctypes.data, nthreads, counts.ctypes.data)
        return out, counts
