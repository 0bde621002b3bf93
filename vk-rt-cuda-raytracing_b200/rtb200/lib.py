"""ctypes binding of libcudabvh_b200.so (the C-ABI in include/*.h).

The library is the product; this module only declares its signatures and
wraps the handles.  It raises if the shared library is missing: there is no
fallback path.  Device buffers are torch CUDA tensors (plumbing only); their
data_ptr() is what crosses the C-ABI.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

import numpy as np

from .scenes import HIT_DTYPE, RAY_DTYPE

PKG_ROOT = Path(__file__).resolve().parent.parent
LIB_PATH = PKG_ROOT / "lib" / "libcudabvh_b200.so"
INCLUDE_DIR = PKG_ROOT.parent / "include"

_lib = None


class RtError(RuntimeError):
    pass


class RtBuildStats(C.Structure):
    _fields_ = [("num_tris", C.c_int), ("num_bvh2_nodes", C.c_int), ("num_nodes", C.c_int), ("depth", C.c_int),
                ("max_leaf", C.c_int), ("bins", C.c_int), ("build_ms", C.c_float), ("sah_cost", C.c_float),
                ("node_bytes", C.c_uint64), ("tri_bytes", C.c_uint64)]


class RtRayGen(C.Structure):
    _fields_ = [("kind", C.c_int), ("count", C.c_int), ("seed", C.c_uint32), ("eps", C.c_float),
                ("tmin", C.c_float), ("tmax", C.c_float), ("light_center", C.c_float * 3),
                ("light_size", C.c_float)]


RT_GEN_DIFFUSE, RT_GEN_SHADOW = 0, 1
RT_BATCH_BUILD_HOST_LOOP = 1  # rtBatch_buildEx: host-driven level loop
RT_REGROUP_MORTON, RT_REGROUP_OCTANT_MORTON = 0, 1


def regroup_rays(d_in, n: int, box6, d_out, kind: int = RT_REGROUP_OCTANT_MORTON, key_bits: int = 32, d_perm=None,
                 stream=None):
    """rtRays_regroup: d_out = d_in reordered by (octant,) origin Morton key; stable."""
    box = np.ascontiguousarray(box6, dtype=np.float32)
    _check(load().rtRays_regroup(_ptr(d_in), n, box.ctypes.data, kind, key_bits, _ptr(d_out),
                                 _ptr(d_perm) if d_perm is not None else None, _stream(stream)), "rtRays_regroup")


class RtInstance(C.Structure):
    _fields_ = [("xform", C.c_float * 12), ("blas", C.c_int32), ("mask", C.c_uint32), ("custom", C.c_uint32),
                ("pad", C.c_uint32)]


class RtMaterial(C.Structure):
    _fields_ = [("albedo", C.c_float * 3), ("emission", C.c_float * 3)]


class RtCamera(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("target", C.c_float * 3), ("up", C.c_float * 3), ("vfov_deg", C.c_float)]


class RtPTParams(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("spp", C.c_int), ("max_bounces", C.c_int),
                ("rr_start", C.c_int), ("seed", C.c_uint32)]


class RtPTStats(C.Structure):
    _fields_ = [("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("light_tris", C.c_int),
                ("light_area", C.c_double)]


class RtBatchTuning(C.Structure):
    _fields_ = [("warps_per_sm", C.c_int), ("node_iters", C.c_int), ("block", C.c_int), ("shared_stack", C.c_int)]


class RtGeometry(C.Structure):
    _fields_ = [("d_vertices", C.c_void_p), ("vertex_stride", C.c_uint64), ("vertex_format", C.c_int),
                ("max_vertex", C.c_int), ("d_indices", C.c_void_p), ("index_type", C.c_int),
                ("num_triangles", C.c_int), ("transform", C.c_void_p)]


RT_VERTEX_FLOAT3, RT_VERTEX_HALF3 = 0, 1
RT_INDEX_NONE, RT_INDEX_UINT16, RT_INDEX_UINT32 = 0, 1, 2


class RtServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("pool_bytes", C.c_uint64), ("max_inflight", C.c_int),
                ("wave_rays", C.c_int), ("chunk_rays", C.c_int), ("max_waves", C.c_int), ("prefetch_rays", C.c_int)]


class RtRequestInfo(C.Structure):
    _fields_ = [("submit_us", C.c_double), ("admit_us", C.c_double), ("done_us", C.c_double), ("status", C.c_int),
                ("waves", C.c_int)]


class RtServerStats(C.Structure):
    _fields_ = [("requests_done", C.c_uint64), ("rays_done", C.c_uint64), ("waves", C.c_uint64),
                ("resident_bytes", C.c_uint64), ("pool_bytes", C.c_uint64), ("peak_pool_used", C.c_uint64),
                ("num_scenes", C.c_int)]


def declared_symbols() -> list[str]:
    """Function names declared in include/*.h."""
    names = []
    for h in sorted(INCLUDE_DIR.glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "defined") and not name.startswith("__"):
                names.append(name)
    return sorted(set(names))


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    global _lib
    if _lib is not None and path is None:
        return _lib
    # RTB200_LIB: another build of the library (an A/B of build options)
    p = Path(path) if path else Path(os.environ.get("RTB200_LIB") or LIB_PATH)
    if not p.exists():
        raise RtError(f"libcudabvh_b200.so not built: {p} (run __graft_entry__.build())")
    L = C.CDLL(str(p))
    vp, i32, f32, u64 = C.c_void_p, C.c_int, C.c_float, C.c_uint64
    sig = {
        "rtGetLastError": (C.c_char_p, []),
        "cudaBVH_build": (vp, [vp, i32]),
        "cudaBVH_buildDevice": (vp, [vp, i32, vp]),
        "cudaBVH_buildFromAABBs": (vp, [vp, i32]),
        "cudaBVH_destroy": (None, [vp]),
        "cudaBVH_traceClosest": (i32, [vp, vp, i32, vp, vp]),
        "cudaBVH_traceAny": (i32, [vp, vp, i32, vp, vp]),
        "cudaBVH_traceClosestHost": (i32, [vp, vp, i32, vp]),
        "cudaBVH_traceAnyHost": (i32, [vp, vp, i32, vp]),
        "cudaBVH_traceClosestHostMulti": (i32, [vp, i32, vp, i32, vp]),
        "cudaBVH_traceAnyHostMulti": (i32, [vp, i32, vp, i32, vp]),
        "cudaBVH_traceCounters": (i32, [vp, vp, i32, i32, vp, vp]),
        "cudaBVH_traceClosestHostNoAlloc": (i32, [vp, vp, i32, vp, vp]),
        "cudaBVH_getStatus": (i32, [vp, vp]),
        "cudaBVH_generateRays": (i32, [vp, vp, vp, i32, C.POINTER(RtRayGen), vp, vp, vp, vp]),
        "rtRays_regroup": (i32, [vp, i32, vp, i32, i32, vp, vp, vp]),
        "rtPT_setRegroup": (i32, [vp, i32, i32]),
        "rtPT_setQueueCapacity": (i32, [vp, C.c_int64]),
        "rtPT_autotune": (i32, [vp, C.POINTER(RtCamera), C.POINTER(RtPTParams), vp, vp, C.POINTER(C.c_int64)]),
        "rtDebug_failAllocations": (i32, [i32]),
        "rtDebug_batchGroups": (i32, [vp, i32, vp, i32]),
        "rtProbe_readBandwidth": (i32, [C.c_uint64, i32, C.POINTER(f32)]),
        "cudaBVH_validate": (i32, [vp]),
        "cudaBVH_getBuildStats": (i32, [vp, C.POINTER(RtBuildStats)]),
        "cudaBVH_getDeviceLayout": (i32, [vp, C.POINTER(vp), C.POINTER(i32), C.POINTER(vp), C.POINTER(i32)]),
        "cudaBVH_tracePrimary": (f32, [vp, i32, f32, f32, f32, vp]),
        "cudaBVH_traceDiffuse": (f32, [vp, i32, vp, vp, vp, vp, vp, vp, vp]),
        "cudaBVH_traceToRGBA": (i32, [vp, i32, i32, f32, f32, f32, vp]),
        "cudaBVH_traceToGPUPtr": (i32, [vp, i32, i32, f32, f32, f32, vp, i32]),
        "cudaBVH_traceToGPUAsync": (None, [vp, i32, i32, f32, f32, f32, vp, i32]),
        "cudaBVH_traceToHostPtr": (i32, [vp, i32, i32, f32, f32, f32, vp, i32, u64]),
        "cudaBVH_importBufferFd": (vp, [i32, u64]),
        "cudaBVH_readGPUMemoryFd": (i32, [i32, u64, u64, u64, vp]),
        "cudaBVH_getBounds": (None, [vp] + [C.POINTER(f32)] * 4),
        "cudaBVH_getNumTris": (i32, [vp]),
        "cudaBVH_getNumBVH4Nodes": (i32, [vp]),
        "cudaBVH_getNumCWBVHNodes": (i32, [vp]),
        "cudaBVH_getNodeData": (vp, [vp]),
        "cudaBVH_getTriData": (None, [vp, vp]),
        "cudaBVH_getStacklessBVH2": (i32, [vp, C.POINTER(C.POINTER(C.c_uint32))]),
        "cudaBVH_getPackedTris": (i32, [vp, C.POINTER(C.POINTER(C.c_float))]),
        "cudaBVH_resetDevice": (None, []),
        "cudaBVH_buildTLASFast": (i32, [vp, i32, C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.POINTER(C.c_int))]),
        "cudaTLAS_build": (vp, [vp, i32, vp, i32]),
        "cudaTLAS_destroy": (None, [vp]),
        "cudaTLAS_traceClosest": (i32, [vp, vp, i32, vp, vp, vp]),
        "cudaTLAS_traceAny": (i32, [vp, vp, i32, vp, vp]),
        "cudaTLAS_getInverseTransforms": (i32, [vp, vp, i32]),
        "cudaTLAS_setTransforms": (i32, [vp, vp, i32]),
        "cudaTLAS_getStatus": (i32, [vp, vp]),
        "rtBatch_build": (vp, [vp, vp, i32, vp]),
        "rtBatch_buildEx": (vp, [vp, vp, i32, i32, vp]),
        "rtBatch_destroy": (None, [vp]),
        "rtBatch_traceClosest": (i32, [vp, vp, vp, i32, vp, vp]),
        "rtBatch_traceAny": (i32, [vp, vp, vp, i32, vp, vp]),
        "rtBatch_traceGraph": (i32, [vp, vp, vp, i32, vp, i32, vp]),
        "rtBatch_autotune": (i32, [vp, vp, vp, i32, vp, vp, C.POINTER(i32), C.POINTER(i32)]),
        "rtBatch_setTuning": (i32, [vp, i32, i32]),
        "rtBatch_setTuningEx": (i32, [vp, C.POINTER(RtBatchTuning)]),
        "rtBatch_getTuning": (i32, [vp, C.POINTER(RtBatchTuning)]),
        "rtBatch_getInfo": (i32, [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(f32)]),
        "rtBatch_getDeviceLayout": (i32, [vp, C.POINTER(vp), C.POINTER(i32), C.POINTER(vp), C.POINTER(i32)]),
        "cudaBVH_buildGeometries": (vp, [C.POINTER(RtGeometry), i32, vp]),
        "cudaBVH_refit": (i32, [vp, vp, vp]),
        "cudaBVH_refitGeometries": (i32, [vp, C.POINTER(RtGeometry), i32, vp]),
        "cudaBVH_serialize": (i32, [vp, vp, C.c_uint64, C.POINTER(C.c_uint64)]),
        "cudaBVH_deserialize": (vp, [vp, C.c_uint64]),
        "rtServer_create": (vp, [C.POINTER(RtServerConfig)]),
        "rtServer_addScene": (i32, [vp, vp]),
        "rtServer_submit": (i32, [vp, i32, i32, vp, i32, vp, C.POINTER(C.c_uint64)]),
        "rtServer_submitDevice": (i32, [vp, i32, i32, vp, i32, vp, C.POINTER(C.c_uint64)]),
        "rtServer_wait": (i32, [vp, C.c_uint64, i32, C.POINTER(RtRequestInfo)]),
        "rtServer_getStats": (i32, [vp, C.POINTER(RtServerStats)]),
        "rtServer_destroy": (None, [vp]),
        "rtPT_create": (vp, [vp, vp, i32, vp]),
        "rtPT_render": (i32, [vp, C.POINTER(RtCamera), C.POINTER(RtPTParams), vp, vp]),
        "rtPT_getStats": (i32, [vp, C.POINTER(RtPTStats)]),
        "rtPT_destroy": (None, [vp]),
        "rtPT_cameraBasis": (i32, [C.POINTER(RtCamera), i32, i32, vp]),
    }
    for name, (res, args) in sig.items():
        if not hasattr(L, name):
            continue  # test_abi checks completeness against the headers
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = L
    return L


def read_bandwidth_gbs(nbytes: int, reps: int = 20) -> float:
    """rtProbe_readBandwidth: streamed read GB/s over an nbytes device buffer."""
    v = C.c_float()
    _check(load().rtProbe_readBandwidth(nbytes, reps, C.byref(v)), "rtProbe_readBandwidth")
    return float(v.value)


def batch_groups(tri_offsets) -> list[int]:
    """Scene-group boundaries rtBatch_build would use for these triangle
    offsets (rtDebug_batchGroups; host only)."""
    off = np.ascontiguousarray(tri_offsets, np.int32)
    out = np.zeros(9, np.int32)
    g = load().rtDebug_batchGroups(off.ctypes.data, len(off) - 1, out.ctypes.data, 8)
    if g < 0:
        raise RtError(f"rtDebug_batchGroups: {last_error()}")
    return out[:g + 1].tolist()


def last_error() -> str:
    return load().rtGetLastError().decode()


def _check(rc: int, what: str):
    if rc != 0:
        raise RtError(f"{what} failed ({rc}): {last_error()}")


def _ptr(x) -> int:
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return int(x)


def _stream(stream) -> int | None:
    if stream is None:
        return None
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


class BVH:
    """A BLAS: cudaBVH_build (host triangles) or cudaBVH_buildDevice."""

    def __init__(self, tris=None, *, device_tris=None, n: int | None = None, stream=None, handle=None):
        L = load()
        if handle is not None:
            self.h = handle
        elif device_tris is not None:
            self.h = L.cudaBVH_buildDevice(_ptr(device_tris), int(n), _stream(stream))
        else:
            tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
            self.h = L.cudaBVH_build(tris.ctypes.data, tris.shape[0])
        if not self.h:
            raise RtError(f"build failed: {last_error()}")

    @classmethod
    def from_geometries(cls, geoms, stream=None) -> "BVH":
        """geoms: list of RtGeometry (device pointers inside)."""
        arr = (RtGeometry * len(geoms))(*geoms)
        h = load().cudaBVH_buildGeometries(arr, len(geoms), _stream(stream))
        if not h:
            raise RtError(f"cudaBVH_buildGeometries failed: {last_error()}")
        return cls(handle=h)

    def refit(self, d_tris, stream=None):
        _check(load().cudaBVH_refit(self.h, _ptr(d_tris), _stream(stream)), "cudaBVH_refit")

    def refit_geometries(self, geoms, stream=None):
        arr = (RtGeometry * len(geoms))(*geoms)
        _check(load().cudaBVH_refitGeometries(self.h, arr, len(geoms), _stream(stream)), "cudaBVH_refitGeometries")

    def serialize(self) -> bytes:
        L = load()
        n = C.c_uint64()
        _check(L.cudaBVH_serialize(self.h, None, 0, C.byref(n)), "cudaBVH_serialize")
        buf = (C.c_ubyte * n.value)()
        _check(L.cudaBVH_serialize(self.h, buf, n.value, C.byref(n)), "cudaBVH_serialize")
        return bytes(buf)

    @classmethod
    def deserialize(cls, blob: bytes) -> "BVH":
        h = load().cudaBVH_deserialize(blob, len(blob))
        if not h:
            raise RtError(f"cudaBVH_deserialize failed: {last_error()}")
        return cls(handle=h)

    @classmethod
    def from_aabbs(cls, aabbs: np.ndarray) -> "BVH":
        a = np.ascontiguousarray(aabbs, dtype=np.float32).reshape(-1, 6)
        h = load().cudaBVH_buildFromAABBs(a.ctypes.data, a.shape[0])
        if not h:
            raise RtError(f"build failed: {last_error()}")
        return cls(handle=h)

    def close(self):
        if getattr(self, "h", None):
            load().cudaBVH_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- traversal on device buffers --
    def closest(self, d_rays, n: int, d_hits, stream=None):
        _check(load().cudaBVH_traceClosest(self.h, _ptr(d_rays), n, _ptr(d_hits), _stream(stream)),
               "cudaBVH_traceClosest")

    def any(self, d_rays, n: int, d_occ, stream=None):
        _check(load().cudaBVH_traceAny(self.h, _ptr(d_rays), n, _ptr(d_occ), _stream(stream)), "cudaBVH_traceAny")

    def generate_rays(self, d_rays, d_hits, n: int, d_out, d_count, kind: int = RT_GEN_DIFFUSE, count: int = 0,
                      seed: int = 3, eps: float = 1e-3, tmin: float = 1e-3, tmax: float = 1e30,
                      light_center=(0.0, 80.0, 0.0), light_size: float = 1.0, d_src=None, stream=None):
        """cudaBVH_generateRays: next-bounce rays from a closest-hit batch (device buffers)."""
        g = RtRayGen(kind, count, seed & 0xFFFFFFFF, eps, tmin, tmax, (C.c_float * 3)(*light_center), light_size)
        _check(load().cudaBVH_generateRays(self.h, _ptr(d_rays), _ptr(d_hits), n, C.byref(g), _ptr(d_out),
                                           _ptr(d_src) if d_src is not None else None, _ptr(d_count),
                                           _stream(stream)), "cudaBVH_generateRays")

    def status(self, stream=None) -> int:
        """cudaBVH_getStatus: RT_OK or RT_ERR_STACK for the device-pointer traces so far."""
        return load().cudaBVH_getStatus(self.h, _stream(stream))

    def counters(self, d_rays, n: int, d_counts, any_hit: bool = False, stream=None):
        _check(load().cudaBVH_traceCounters(self.h, _ptr(d_rays), n, int(any_hit), _ptr(d_counts), _stream(stream)),
               "cudaBVH_traceCounters")

    # -- traversal on host buffers --
    def closest_host(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
        hits = np.zeros(rays.shape[0], dtype=HIT_DTYPE)
        _check(load().cudaBVH_traceClosestHost(self.h, rays.ctypes.data, rays.shape[0], hits.ctypes.data),
               "cudaBVH_traceClosestHost")
        return hits

    def any_host(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
        occ = np.zeros(rays.shape[0], dtype=np.uint8)
        _check(load().cudaBVH_traceAnyHost(self.h, rays.ctypes.data, rays.shape[0], occ.ctypes.data),
               "cudaBVH_traceAnyHost")
        return occ

    # -- introspection / exports --
    def validate(self):
        _check(load().cudaBVH_validate(self.h), "cudaBVH_validate")

    def stats(self) -> dict:
        s = RtBuildStats()
        _check(load().cudaBVH_getBuildStats(self.h, C.byref(s)), "cudaBVH_getBuildStats")
        return {f: getattr(s, f) for f, _ in RtBuildStats._fields_}

    def layout(self):
        n_nodes, n_tris = C.c_int(), C.c_int()
        pn, pt = C.c_void_p(), C.c_void_p()
        _check(load().cudaBVH_getDeviceLayout(self.h, C.byref(pn), C.byref(n_nodes), C.byref(pt), C.byref(n_tris)),
               "cudaBVH_getDeviceLayout")
        return pn.value, n_nodes.value, pt.value, n_tris.value

    def bounds(self):
        f = [C.c_float() for _ in range(4)]
        load().cudaBVH_getBounds(self.h, *[C.byref(x) for x in f])
        return np.array([x.value for x in f], np.float32)

    def exports(self) -> dict:
        L = load()
        pd = C.POINTER(C.c_uint32)()
        nd = L.cudaBVH_getStacklessBVH2(self.h, C.byref(pd))
        pp = C.POINTER(C.c_float)()
        npk = L.cudaBVH_getPackedTris(self.h, C.byref(pp))
        nb4 = L.cudaBVH_getNumBVH4Nodes(self.h)
        b4p = L.cudaBVH_getNodeData(self.h)
        ptrs = (C.c_void_p * 9)()
        L.cudaBVH_getTriData(self.h, C.byref(ptrs))
        ntri = L.cudaBVH_getNumTris(self.h)
        return {
            "dfs": np.ctypeslib.as_array(pd, shape=(nd * 8,)).copy() if nd else np.zeros(0, np.uint32),
            "packed": np.ctypeslib.as_array(pp, shape=(npk * 4,)).copy() if npk else np.zeros(0, np.float32),
            "bvh4": np.frombuffer(C.string_at(b4p, nb4 * 64), np.uint8).copy() if nb4 else np.zeros(0, np.uint8),
            "soa": np.stack([np.ctypeslib.as_array(C.cast(ptrs[i], C.POINTER(C.c_float)), shape=(ntri,)).copy()
                             for i in range(9)]),
            "num_cwbvh": L.cudaBVH_getNumCWBVHNodes(self.h),
        }

    # -- reference-shaped traces --
    def trace_primary(self, side: int, cam, want_t: bool = True):
        t = np.zeros(side * side, np.float32) if want_t else None
        mrs = load().cudaBVH_tracePrimary(self.h, side, float(cam[0]), float(cam[1]), float(cam[2]),
                                          t.ctypes.data if want_t else None)
        return mrs, t

    def trace_diffuse(self, org: np.ndarray, dirs: np.ndarray):
        n = org.shape[0]
        cols = [np.ascontiguousarray(org[:, k], np.float32) for k in range(3)] + \
               [np.ascontiguousarray(dirs[:, k], np.float32) for k in range(3)]
        t = np.zeros(n, np.float32)
        mrs = load().cudaBVH_traceDiffuse(self.h, n, *[c.ctypes.data for c in cols], t.ctypes.data)
        return mrs, t

    def trace_rgba(self, w: int, h: int, cam) -> np.ndarray:
        out = np.zeros(w * h, np.uint32)
        _check(load().cudaBVH_traceToRGBA(self.h, w, h, float(cam[0]), float(cam[1]), float(cam[2]),
                                          out.ctypes.data), "cudaBVH_traceToRGBA")
        return out


def tlas_fast(aabbs: np.ndarray):
    a = np.ascontiguousarray(aabbs, dtype=np.float32).reshape(-1, 6)
    L = load()
    pn = C.POINTER(C.c_uint32)()
    po = C.POINTER(C.c_int)()
    m = L.cudaBVH_buildTLASFast(a.ctypes.data, a.shape[0], C.byref(pn), C.byref(po))
    if m <= 0:
        return np.zeros(0, np.uint32), np.zeros(0, np.int32)
    nodes = np.ctypeslib.as_array(pn, shape=(m * 8,)).copy()
    ordered = np.ctypeslib.as_array(po, shape=(a.shape[0],)).copy()
    libc = C.CDLL("libc.so.6")
    libc.free(C.cast(pn, C.c_void_p))
    libc.free(C.cast(po, C.c_void_p))
    return nodes, ordered


def trace_host_multi(bvhs, rays: np.ndarray, any_hit: bool = False) -> np.ndarray:
    """cudaBVH_traceClosestHostMulti / cudaBVH_traceAnyHostMulti: one host
    batch split over replicas of a scene (one BVH per GPU)."""
    rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
    hs = (C.c_void_p * len(bvhs))(*[b.h for b in bvhs])
    if any_hit:
        out = np.zeros(rays.shape[0], dtype=np.uint8)
        _check(load().cudaBVH_traceAnyHostMulti(hs, len(bvhs), rays.ctypes.data, rays.shape[0], out.ctypes.data),
               "cudaBVH_traceAnyHostMulti")
    else:
        out = np.zeros(rays.shape[0], dtype=HIT_DTYPE)
        _check(load().cudaBVH_traceClosestHostMulti(hs, len(bvhs), rays.ctypes.data, rays.shape[0],
                                                    out.ctypes.data), "cudaBVH_traceClosestHostMulti")
    return out


class TLAS:
    """cudaTLAS_build over BVH handles and 3x4 instance transforms."""

    def __init__(self, blases, xforms: np.ndarray, blas_index: np.ndarray):
        L = load()
        self.blases = list(blases)
        n = len(blas_index)
        self.instances = (RtInstance * n)()
        for k in range(n):
            self.instances[k].xform[:] = np.asarray(xforms[k], np.float32).ravel().tolist()
            self.instances[k].blas = int(blas_index[k])
        arr = (C.c_void_p * len(self.blases))(*[b.h for b in self.blases])
        self.h = L.cudaTLAS_build(arr, len(self.blases), self.instances, n)
        if not self.h:
            raise RtError(f"cudaTLAS_build failed: {last_error()}")
        self.n = n

    def set_transforms(self, xforms: np.ndarray, blas_index: np.ndarray):
        """cudaTLAS_setTransforms: new instance transforms / BLAS choices, same count."""
        inst = (RtInstance * self.n)()
        for k in range(self.n):
            inst[k].xform[:] = np.asarray(xforms[k], np.float32).ravel().tolist()
            inst[k].blas = int(blas_index[k])
        _check(load().cudaTLAS_setTransforms(self.h, inst, self.n), "cudaTLAS_setTransforms")
        self.instances = inst

    def inverse(self) -> np.ndarray:
        out = np.zeros((self.n, 12), np.float32)
        _check(load().cudaTLAS_getInverseTransforms(self.h, out.ctypes.data, self.n), "getInverseTransforms")
        return out

    def closest(self, d_rays, n, d_hits, d_inst=None, stream=None):
        _check(load().cudaTLAS_traceClosest(self.h, _ptr(d_rays), n, _ptr(d_hits),
                                            _ptr(d_inst) if d_inst is not None else None, _stream(stream)),
               "cudaTLAS_traceClosest")

    def any(self, d_rays, n, d_occ, stream=None):
        _check(load().cudaTLAS_traceAny(self.h, _ptr(d_rays), n, _ptr(d_occ), _stream(stream)), "cudaTLAS_traceAny")

    def close(self):
        if getattr(self, "h", None):
            load().cudaTLAS_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_camera(eye, target, up=(0.0, 1.0, 0.0), vfov=45.0) -> RtCamera:
    c = RtCamera()
    c.eye[:] = list(map(float, eye))
    c.target[:] = list(map(float, target))
    c.up[:] = list(map(float, up))
    c.vfov_deg = float(vfov)
    return c


def camera_basis(cam: RtCamera, w: int, h: int) -> np.ndarray:
    out = np.zeros(14, np.float32)
    _check(load().rtPT_cameraBasis(C.byref(cam), w, h, out.ctypes.data), "rtPT_cameraBasis")
    return out


class PathTracer:
    """rtPT_create / rtPT_render over a TLAS."""

    def __init__(self, tlas: TLAS, albedo: np.ndarray, emission: np.ndarray):
        n = tlas.n
        self.mats = (RtMaterial * n)()
        for k in range(n):
            self.mats[k].albedo[:] = np.asarray(albedo[k], np.float32).tolist()
            self.mats[k].emission[:] = np.asarray(emission[k], np.float32).tolist()
        self.tlas = tlas
        self.h = load().rtPT_create(tlas.h, self.mats, n, tlas.instances)
        if not self.h:
            raise RtError(f"rtPT_create failed: {last_error()}")

    def render(self, cam: RtCamera, w: int, h: int, spp: int, max_bounces: int = 4, rr_start: int = 2,
               seed: int = 1, d_rgb=None, stream=None):
        p = RtPTParams(w, h, spp, max_bounces, rr_start, seed)
        _check(load().rtPT_render(self.h, C.byref(cam), C.byref(p), _ptr(d_rgb), _stream(stream)), "rtPT_render")

    def set_queue_capacity(self, paths: int):
        """rtPT_setQueueCapacity: paths per slice (0 = the whole frame)."""
        _check(load().rtPT_setQueueCapacity(self.h, paths), "rtPT_setQueueCapacity")

    def autotune(self, cam, w: int, h: int, spp: int, max_bounces: int = 4, rr_start: int = 2, seed: int = 1,
                 d_rgb=None, stream=None) -> int:
        """rtPT_autotune: the fastest queue capacity for this frame (0 = whole frame)."""
        prm = RtPTParams(w, h, spp, max_bounces, rr_start, seed)
        out = C.c_int64()
        _check(load().rtPT_autotune(self.h, C.byref(cam), C.byref(prm), _ptr(d_rgb), _stream(stream), C.byref(out)),
               "rtPT_autotune")
        return int(out.value)

    def set_regroup(self, key_bits: int, kind: int = RT_REGROUP_OCTANT_MORTON):
        """rtPT_setRegroup: regroup bounce rays before each extension trace (0 = off)."""
        _check(load().rtPT_setRegroup(self.h, kind, key_bits), "rtPT_setRegroup")

    def stats(self) -> dict:
        s = RtPTStats()
        _check(load().rtPT_getStats(self.h, C.byref(s)), "rtPT_getStats")
        return {f: getattr(s, f) for f, _ in RtPTStats._fields_}

    def close(self):
        if getattr(self, "h", None):
            load().rtPT_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """rtBatch_*: many scenes built and traced together."""

    def __init__(self, scenes_tris=None, stream=None, *, all_tris=None, tri_offsets=None, host_loop=False):
        """scenes_tris: list of (n_i, 9) arrays; or all_tris (sum n_i, 9) with
        tri_offsets (num_scenes + 1) already concatenated.  host_loop: build
        with the host-driven level loop instead of the one-graph build."""
        L = load()
        if all_tris is None:
            tris = [np.ascontiguousarray(t, np.float32).reshape(-1, 9) for t in scenes_tris]
            tri_offsets = np.concatenate([[0], np.cumsum([t.shape[0] for t in tris])])
            all_tris = np.concatenate(tris)
        self.tri_off = np.ascontiguousarray(tri_offsets, np.int32)
        allt = np.ascontiguousarray(all_tris, np.float32).reshape(-1, 9)
        self.h = L.rtBatch_buildEx(allt.ctypes.data, self.tri_off.ctypes.data, len(self.tri_off) - 1,
                                   RT_BATCH_BUILD_HOST_LOOP if host_loop else 0, _stream(stream))
        if not self.h:
            raise RtError(f"rtBatch_build failed: {last_error()}")
        self.num_scenes = len(self.tri_off) - 1

    def info(self):
        a, b, c = C.c_int(), C.c_int(), C.c_float()
        _check(load().rtBatch_getInfo(self.h, C.byref(a), C.byref(b), C.byref(c)), "rtBatch_getInfo")
        return {"num_scenes": a.value, "num_nodes": b.value, "build_ms": c.value}

    def layout(self):
        """(nodes pointer, node count, triangle-record pointer, record count) on the device."""
        n_nodes, n_tris = C.c_int(), C.c_int()
        pn, pt = C.c_void_p(), C.c_void_p()
        _check(load().rtBatch_getDeviceLayout(self.h, C.byref(pn), C.byref(n_nodes), C.byref(pt), C.byref(n_tris)),
               "rtBatch_getDeviceLayout")
        return pn.value, n_nodes.value, pt.value, n_tris.value

    def closest(self, d_rays, d_off, n, d_hits, stream=None):
        _check(load().rtBatch_traceClosest(self.h, _ptr(d_rays), _ptr(d_off), n, _ptr(d_hits), _stream(stream)),
               "rtBatch_traceClosest")

    def any(self, d_rays, d_off, n, d_occ, stream=None):
        _check(load().rtBatch_traceAny(self.h, _ptr(d_rays), _ptr(d_off), n, _ptr(d_occ), _stream(stream)),
               "rtBatch_traceAny")

    def graph(self, d_rays, d_off, n, d_out, any_hit=False, stream=None):
        _check(load().rtBatch_traceGraph(self.h, _ptr(d_rays), _ptr(d_off), n, _ptr(d_out), int(any_hit),
                                         _stream(stream)), "rtBatch_traceGraph")

    def autotune(self, d_rays, d_off, n, d_hits, stream=None):
        c, it = C.c_int(), C.c_int()
        _check(load().rtBatch_autotune(self.h, _ptr(d_rays), _ptr(d_off), n, _ptr(d_hits), _stream(stream),
                                       C.byref(c), C.byref(it)), "rtBatch_autotune")
        return c.value, it.value

    def set_tuning(self, ctas, iters):
        _check(load().rtBatch_setTuning(self.h, ctas, iters), "rtBatch_setTuning")

    def tuning(self) -> dict:
        """rtBatch_getTuning: the launch shape in use."""
        t = RtBatchTuning()
        _check(load().rtBatch_getTuning(self.h, C.byref(t)), "rtBatch_getTuning")
        return {f: getattr(t, f) for f, _ in RtBatchTuning._fields_}

    def set_tuning_ex(self, warps_per_sm: int, node_iters: int, block: int, shared_stack: int):
        t = RtBatchTuning(warps_per_sm, node_iters, block, shared_stack)
        _check(load().rtBatch_setTuningEx(self.h, C.byref(t)), "rtBatch_setTuningEx")

    def close(self):
        if getattr(self, "h", None):
            load().rtBatch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """rtServer_*: resident scenes, requests admitted by footprint and traced
    in shared wavefronts by the library's scheduler thread."""

    def __init__(self, hbm_budget_bytes=0, pool_bytes=0, max_inflight=0, wave_rays=0, chunk_rays=0, max_waves=0,
                 prefetch_rays=0):
        cfg = RtServerConfig(hbm_budget_bytes, pool_bytes, max_inflight, wave_rays, chunk_rays, max_waves,
                             prefetch_rays)
        self.h = load().rtServer_create(C.byref(cfg))
        if not self.h:
            raise RtError(f"rtServer_create failed: {last_error()}")

    def add_scene(self, bvh: "BVH") -> int:
        rc = load().rtServer_addScene(self.h, bvh.h)
        if rc < 0:
            raise RtError(f"rtServer_addScene failed ({rc}): {last_error()}")
        return rc

    def submit(self, scene: int, any_hit: bool, rays_ptr: int, n: int, out_ptr: int, device: bool = False) -> int:
        """Pointers are raw addresses (host for device=False, device otherwise)."""
        t = C.c_uint64()
        f = load().rtServer_submitDevice if device else load().rtServer_submit
        _check(f(self.h, scene, int(any_hit), rays_ptr, n, out_ptr, C.byref(t)), "rtServer_submit")
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> dict:
        info = RtRequestInfo()
        rc = load().rtServer_wait(self.h, ticket, timeout_ms, C.byref(info))
        if rc != 0:
            raise RtError(f"rtServer_wait: {rc}: {last_error()}")
        return {"submit_us": info.submit_us, "admit_us": info.admit_us, "done_us": info.done_us,
                "status": info.status, "waves": info.waves}

    def stats(self) -> dict:
        st = RtServerStats()
        _check(load().rtServer_getStats(self.h, C.byref(st)), "rtServer_getStats")
        return {k: getattr(st, k) for k, _ in RtServerStats._fields_}

    def close(self):
        if getattr(self, "h", None):
            load().rtServer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
