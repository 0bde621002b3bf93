"""Seeded procedural scenes and ray batches for the five workloads.

Every draw comes from Philox4x32-10 keyed by (seed, stream id), so a scene or
ray batch is a pure function of its arguments.  Geometry is float32 AoS
triangles, 9 floats each (the reference's CudaTri, layer/cuda_bvh_backend.h:16-18).

Workloads (sizes as stated for them):
  primary_1080p_100k   200 UV spheres x 500 tris in a 100^3 box + 2-tri ground
                       plane = 100,002 tris; 1920x1080 pinhole, 1 ray/pixel.
  incoherent_2m        random sphere/box meshes of 1K-20K tris (log-uniform)
                       until 2,000,000 tris; rays = 2M cosine-weighted diffuse
                       bounces (closest hit) + 2M shadow rays to a 1x1 area
                       light (any hit) from the 1080p camera's hit points.
  pathtrace_tlas_5m    16 BLASes totalling 5M tris, 64 instances with random
                       affine transforms; Lambertian albedo U[0.1,0.9],
                       5% emissive instances with radiance U[1,20].
  batched_256          256 scenes, seeds 0..255, tris log-uniform 1K-500K.
  served_16            16 resident scenes, tris log-uniform 200K-5M.
"""
from __future__ import annotations

import concurrent.futures
import functools
import math
import os

import numpy as np

from .philox import uniforms

RAY_DTYPE = np.dtype([("org", "<f4", 3), ("tmin", "<f4"), ("dir", "<f4", 3), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("prim", "<i4"), ("u", "<f4"), ("v", "<f4")])

# Philox stream ids (second key word) for the different draws.
S_PLACE, S_MESH, S_DIFFUSE, S_SHADOW, S_INST, S_MAT, S_BATCH, S_SERVE = 1, 2, 3, 4, 5, 6, 7, 8

F32 = np.float32


# ------------------------------------------------------------------ meshes --
def uv_sphere(segs: int, rings: int) -> np.ndarray:
    """Unit UV sphere: 2*segs*(rings-1) triangles (caps are fans).  Quad
    (r, s) spans rings r..r+1 and segments s..s+1 and gives triangles
    (a, b, c) except on the top ring and (a, c, d) except on the bottom."""
    th = np.linspace(0.0, math.pi, rings + 1)
    ph = np.linspace(0.0, 2.0 * math.pi, segs + 1)
    T, P = np.meshgrid(th, ph, indexing="ij")
    V = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], axis=-1)
    a, b, c, d = V[:-1, :-1], V[:-1, 1:], V[1:, 1:], V[1:, :-1]
    t = np.empty((rings, segs, 2, 3, 3))
    t[:, :, 0] = np.stack([a, b, c], axis=2)
    t[:, :, 1] = np.stack([a, c, d], axis=2)
    keep = np.ones((rings, segs, 2), bool)
    keep[0, :, 0] = False
    keep[rings - 1, :, 1] = False
    return t[keep].reshape(-1, 3, 3)


def box_mesh(m: int) -> np.ndarray:
    """Unit cube [-1,1]^3, each face an m x m grid of quads: 12*m*m triangles,
    faces in (axis, sign) order, quads (i, j) row-major, two triangles per
    quad, winding reversed on the negative faces."""
    g = np.linspace(-1.0, 1.0, m + 1)
    i, j = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    corners = [(i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)]
    out = []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            q = np.zeros((m, m, 4, 3))
            for k, (ca, cb) in enumerate(corners):
                q[:, :, k, axis] = sign
                q[:, :, k, (axis + 1) % 3] = g[ca]
                q[:, :, k, (axis + 2) % 3] = g[cb]
            if sign < 0:
                q = q[:, :, ::-1]
            t = np.stack([q[:, :, [0, 1, 2]], q[:, :, [0, 2, 3]]], axis=2)
            out.append(t.reshape(-1, 3, 3))
    return np.concatenate(out)


@functools.lru_cache(maxsize=None)
def _template(kind: int, ntris: int) -> np.ndarray:
    t = _mesh_of_size(kind, ntris)
    t.setflags(write=False)
    return t


def mesh_of_size(kind: int, ntris: int) -> np.ndarray:
    """Sphere (kind 0) or box (kind 1) template with about `ntris` triangles
    (templates are cached; the result is read-only)."""
    return _template(kind, ntris)


def _mesh_of_size(kind: int, ntris: int) -> np.ndarray:
    if kind == 0:
        segs = max(3, int(round(math.sqrt(ntris))))
        rings = max(2, int(round(ntris / (2 * segs))) + 1)
        return uv_sphere(segs, rings)
    m = max(1, int(round(math.sqrt(ntris / 12.0))))
    return box_mesh(m)


def rotations(u: np.ndarray) -> np.ndarray:
    """Uniform random rotations from (n, 3) uniforms (Shoemake's quaternion)."""
    u = u.astype(np.float64)
    a, b, c = u[:, 0], 2 * math.pi * u[:, 1], 2 * math.pi * u[:, 2]
    q = np.stack([np.sqrt(1 - a) * np.sin(b), np.sqrt(1 - a) * np.cos(b),
                  np.sqrt(a) * np.sin(c), np.sqrt(a) * np.cos(c)], axis=1)
    x, y, z, w = q.T
    R = np.empty((u.shape[0], 3, 3))
    R[:, 0] = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], 1)
    R[:, 1] = np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], 1)
    R[:, 2] = np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], 1)
    return R


def ground_plane(y: float, half: float) -> np.ndarray:
    a, b, c, d = [(-half, y, -half), (half, y, -half), (half, y, half), (-half, y, half)]
    return np.asarray([(a, c, b), (a, d, c)], dtype=np.float64)


def log_uniform(u: np.ndarray, lo: float, hi: float) -> np.ndarray:
    return np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))


def _place(tmpl: np.ndarray, R: np.ndarray, s: float, t: np.ndarray) -> np.ndarray:
    return (tmpl.reshape(-1, 3) @ R.T * s + t).reshape(-1, 3, 3)


# ------------------------------------------------------------------ scenes --
def scene_spheres_100k(seed: int = 0, nspheres: int = 200, box: float = 100.0) -> np.ndarray:
    """200 UV spheres of exactly 500 tris (25 segments x 11 rings) placed
    uniformly in a box^3 cube, radius log-uniform [2, 8], random rotation,
    plus a 2-triangle ground plane: (nspheres*500 + 2, 9) float32."""
    tmpl = uv_sphere(25, 11)
    assert tmpl.shape[0] == 500
    u = uniforms(seed, S_PLACE, nspheres, 8)
    R = rotations(u[:, 4:7])
    out = [ground_plane(-0.5 * box - 2.0, 1.5 * box)]
    for i in range(nspheres):
        c = (u[i, 0:3].astype(np.float64) - 0.5) * box
        r = log_uniform(float(u[i, 3]), 2.0, 8.0)
        out.append(_place(tmpl, R[i], r, c))
    return np.concatenate(out).reshape(-1, 9).astype(F32)


def scene_meshes(seed: int, ntris: int, box: float = 100.0, lo: int = 1000, hi: int = 20000,
                 ground: bool = True) -> np.ndarray:
    """Random sphere/box meshes (kinds 50/50) of log-uniform [lo, hi] triangles
    until exactly `ntris` triangles (the last mesh is trimmed); radius
    log-uniform [2, 10] scaled with the box, random rotation, uniform centre."""
    out = []
    total = 0
    if ground:
        out.append(ground_plane(-0.5 * box - 2.0, 1.5 * box))
        total = 2
    i = 0
    scale = box / 100.0
    cap = 0
    while total < ntris:
        if i >= cap:  # item i of a Philox stream does not depend on how many are drawn
            cap = max(64, 2 * cap)
            um, up = uniforms(seed, S_MESH, cap, 8), uniforms(seed, S_PLACE, cap, 4)
        u = um[i]
        k = int(u[0] < 0.5)
        want = int(round(log_uniform(float(u[1]), lo, hi)))
        m = mesh_of_size(k, want)
        R = rotations(u[None, 2:5])[0]
        c = (u[5:8].astype(np.float64) - 0.5) * box
        r = log_uniform(float(up[i, 0]), 2.0, 10.0) * scale
        m = _place(m, R, r, c)
        if total + m.shape[0] > ntris:
            m = m[: ntris - total]
        out.append(m)
        total += m.shape[0]
        i += 1
    return np.concatenate(out).reshape(-1, 9).astype(F32)


# -------------------------------------------------------------------- rays --
def camera_basis(eye, target, up=(0.0, 1.0, 0.0)):
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    return eye, f, r, u


def pinhole_rays(width: int, height: int, eye, target, vfov_deg: float = 45.0,
                 tmin: float = 0.0, tmax: float = 1e30) -> np.ndarray:
    """One ray per pixel centre, row-major from the top-left; directions
    normalised in float64 then stored as float32."""
    eye, f, r, u = camera_basis(eye, target)
    th = math.tan(math.radians(vfov_deg) * 0.5)
    aspect = width / height
    px = (np.arange(width) + 0.5) / width * 2.0 - 1.0
    py = 1.0 - (np.arange(height) + 0.5) / height * 2.0
    X, Y = np.meshgrid(px * th * aspect, py * th)
    d = f[None, None, :] + X[..., None] * r[None, None, :] + Y[..., None] * u[None, None, :]
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    rays = np.zeros(width * height, dtype=RAY_DTYPE)
    rays["org"] = eye.astype(F32)
    rays["dir"] = d.reshape(-1, 3).astype(F32)
    rays["tmin"] = tmin
    rays["tmax"] = tmax
    return rays


CAM_EYE = (0.0, 30.0, -170.0)
CAM_TARGET = (0.0, 0.0, 0.0)


def primary_1080p() -> np.ndarray:
    return pinhole_rays(1920, 1080, CAM_EYE, CAM_TARGET, 45.0)


def hit_frame(tris: np.ndarray, rays: np.ndarray, hits: np.ndarray):
    """Hit points and geometric normals facing the incoming ray (float32)."""
    ok = hits["prim"] >= 0
    r = rays[ok]
    h = hits[ok]
    p = r["org"].astype(F32) + h["t"].astype(F32)[:, None] * r["dir"].astype(F32)
    tv = tris.reshape(-1, 3, 3)[h["prim"]].astype(np.float64)
    n = np.cross(tv[:, 1] - tv[:, 0], tv[:, 2] - tv[:, 0])
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    flip = np.einsum("ij,ij->i", n, r["dir"].astype(np.float64)) > 0
    n[flip] *= -1
    return p.astype(F32), n.astype(F32)


def _onb(n: np.ndarray):
    """Orthonormal tangent frame around unit normals (branch on the larger of |nx|,|ny|)."""
    t = np.zeros_like(n)
    big = np.abs(n[:, 0]) > np.abs(n[:, 1])
    il = 1.0 / np.sqrt(n[big, 0] ** 2 + n[big, 2] ** 2)
    t[big] = np.stack([-n[big, 2] * il, np.zeros(big.sum()), n[big, 0] * il], 1)
    sm = ~big
    il = 1.0 / np.sqrt(n[sm, 1] ** 2 + n[sm, 2] ** 2)
    t[sm] = np.stack([np.zeros(sm.sum()), n[sm, 2] * il, -n[sm, 1] * il], 1)
    b = np.cross(n, t)
    return t, b


def diffuse_rays(points: np.ndarray, normals: np.ndarray, count: int, seed: int,
                 eps: float = 1e-3, tmin: float = 1e-3, tmax: float = 1e30) -> np.ndarray:
    """`count` cosine-weighted bounce rays; ray i leaves hit point i mod len.
    Malley's method on a rejection-sampled unit disk; origin offset eps*n
    (the multi_bounce.cu:355-356 form)."""
    m = points.shape[0]
    src = np.arange(count) % m
    n = normals[src].astype(np.float64)
    u = uniforms(seed, S_DIFFUSE, count, 16).astype(np.float64) * 2.0 - 1.0
    x = np.zeros(count)
    y = np.zeros(count)
    done = np.zeros(count, bool)
    for k in range(8):
        a, b = u[:, 2 * k], u[:, 2 * k + 1]
        take = (~done) & (a * a + b * b < 1.0)
        x[take], y[take] = a[take], b[take]
        done |= take
    z = np.sqrt(np.maximum(0.0, 1.0 - x * x - y * y))
    t, b = _onb(n)
    d = x[:, None] * t + y[:, None] * b + z[:, None] * n
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros(count, dtype=RAY_DTYPE)
    rays["org"] = (points[src].astype(np.float64) + eps * n).astype(F32)
    rays["dir"] = d.astype(F32)
    rays["tmin"] = tmin
    rays["tmax"] = tmax
    return rays


LIGHT_CENTER = (0.0, 80.0, 0.0)


def shadow_rays(points: np.ndarray, normals: np.ndarray, count: int, seed: int,
                light_center=LIGHT_CENTER, light_size: float = 1.0, eps: float = 1e-3) -> np.ndarray:
    """`count` any-hit rays toward a uniform point of a light_size^2 square
    (parallel to xz) centred at light_center; tmax stops just short of it."""
    m = points.shape[0]
    src = np.arange(count) % m
    u = uniforms(seed, S_SHADOW, count, 4).astype(np.float64)
    L = np.asarray(light_center, np.float64)[None, :] + np.stack(
        [(u[:, 0] - 0.5) * light_size, np.zeros(count), (u[:, 1] - 0.5) * light_size], 1)
    o = points[src].astype(np.float64) + eps * normals[src].astype(np.float64)
    d = L - o
    dist = np.linalg.norm(d, axis=1)
    rays = np.zeros(count, dtype=RAY_DTYPE)
    rays["org"] = o.astype(F32)
    rays["dir"] = (d / dist[:, None]).astype(F32)
    rays["tmin"] = 1e-3
    rays["tmax"] = (dist * (1.0 - 1e-4)).astype(F32)
    return rays


def random_rays(seed: int, count: int, box: float = 100.0) -> np.ndarray:
    """Uniform origins in the box and uniform directions: an incoherent mix
    of hits and misses for parity tests."""
    u = uniforms(seed, S_DIFFUSE + 100, count, 8).astype(np.float64)
    o = (u[:, 0:3] - 0.5) * box
    z = 2 * u[:, 3] - 1
    ph = 2 * math.pi * u[:, 4]
    s = np.sqrt(np.maximum(0, 1 - z * z))
    d = np.stack([s * np.cos(ph), s * np.sin(ph), z], 1)
    rays = np.zeros(count, dtype=RAY_DTYPE)
    rays["org"] = o.astype(F32)
    rays["dir"] = d.astype(F32)
    rays["tmin"] = 0.0
    rays["tmax"] = 1e30
    return rays


# ------------------------------------------------------- instanced scenes --
def instanced_scene(seed: int, total_tris: int, nblas: int = 16, ninst: int = 64, world: float = 100.0,
                    emissive_frac: float = 0.05):
    """Instanced path-tracing scene: `nblas` BLASes (clusters of sphere/box meshes in a
    local 12^3 box over a 36 x 36 two-triangle floor) totalling `total_tris` triangles, `ninst` instances with
    random rotation, log-uniform scale [1.5, 5] and uniform translation in
    the world box, Lambertian albedo U[0.1, 0.9] per instance and emission
    U[1, 20] (grey) on ~emissive_frac of the instances (at least one).
    Returns (blas list of (n,9) float32, xforms (ninst,3,4) float32,
    blas index per instance, albedo (ninst,3), emission (ninst,3))."""
    per = total_tris // nblas
    blases = []
    for b in range(nblas):
        n = per if b < nblas - 1 else total_tris - per * (nblas - 1)
        blases.append(scene_meshes(seed * 1000 + b, n, box=12.0, lo=min(1000, n), hi=max(min(20000, n), 1000),
                                   ground=True))
    u = uniforms(seed, S_INST, ninst, 12).astype(np.float64)
    R = rotations(u[:, 0:3])
    sc = log_uniform(u[:, 3], 1.5, 5.0)
    t = (u[:, 4:7] - 0.5) * world
    xf = np.zeros((ninst, 3, 4), np.float32)
    xf[:, :, :3] = (R * sc[:, None, None]).astype(np.float32)
    xf[:, :, 3] = t.astype(np.float32)
    bidx = (np.arange(ninst) % nblas).astype(np.int32)
    m = uniforms(seed, S_MAT, ninst, 8).astype(np.float64)
    albedo = (0.1 + 0.8 * m[:, 0:3]).astype(np.float32)
    emissive = m[:, 3] < emissive_frac
    if not emissive.any():
        emissive[int(np.argmin(m[:, 3]))] = True
    emission = np.zeros((ninst, 3), np.float32)
    emission[emissive] = (1.0 + 19.0 * m[emissive, 4:5]).astype(np.float32)
    return blases, xf, bidx, albedo, emission


PT_CAM_EYE = (0.0, 20.0, -120.0)
PT_CAM_TARGET = (0.0, 0.0, 0.0)


# ---------------------------------------------------------- batched scenes --
def batched_sizes(nscenes: int = 256, tri_lo: int = 1000, tri_hi: int = 500_000, ray_lo: int = 4096,
                  ray_hi: int = 2_000_000, seed: int = 7):
    """Triangle and ray counts of the batched workload's scenes (n_i and
    r_i of batched_workload), without making the scenes."""
    u = uniforms(seed, S_BATCH, nscenes, 4).astype(np.float64)
    ntris = np.round(log_uniform(u[:, 0], tri_lo, tri_hi)).astype(int)
    nrays = np.round(log_uniform(u[:, 1], ray_lo, ray_hi)).astype(int)
    return ntris, nrays


def batched_workload(nscenes: int = 256, tri_lo: int = 1000, tri_hi: int = 500_000, ray_lo: int = 4096,
                     ray_hi: int = 2_000_000, seed: int = 7, scenes=None):
    """Batched workload of 256 scenes: scene i = scene_meshes(seed=i, n_i) with
    n_i log-uniform in [tri_lo, tri_hi]; its ray batch has r_i log-uniform in
    [ray_lo, ray_hi] rays, half primary and half diffuse (scene_rays).
    `scenes` (a range of scene ids, default all) makes only those scenes, the
    same as in the full workload.  Returns (list of (n_i, 9) float32, rays
    concatenated, ray offsets)."""
    ntris, nrays = batched_sizes(nscenes, tri_lo, tri_hi, ray_lo, ray_hi, seed)
    ids = range(nscenes) if scenes is None else scenes
    def one(i):
        t = scene_meshes(i, int(ntris[i]))
        return t, scene_rays(t, int(nrays[i]), seed=i)

    with concurrent.futures.ThreadPoolExecutor(min(16, os.cpu_count() or 1)) as ex:
        res = list(ex.map(one, ids))
    tris, rays = [r[0] for r in res], [r[1] for r in res]
    off = np.concatenate([[0], np.cumsum([r.shape[0] for r in rays])]).astype(np.int32)
    return tris, np.concatenate(rays), off


def scene_rays(tris: np.ndarray, n: int, seed: int) -> np.ndarray:
    """n rays for one scene: n//2 coherent primary rays (row-major pixels of
    a 16:9 pinhole camera in front of the scene's bounds) then n - n//2
    diffuse rays (uniform point on a uniformly chosen triangle, cosine-
    weighted about its face normal by the polar disk map).  Drawn with
    numpy's PCG64 seeded by (seed, 3): cheap enough for tens of millions."""
    v = tris.reshape(-1, 3, 3)
    flat = v.reshape(-1, 3)
    lo, hi = flat.min(0).astype(np.float64), flat.max(0).astype(np.float64)
    c, ext = (lo + hi) / 2, float(np.linalg.norm(hi - lo))
    npri = n // 2
    w = max(16, int(math.ceil(math.sqrt(npri * 16 / 9))))
    h = max(9, int(math.ceil(npri / w)))
    pri = pinhole_rays(w, h, c + np.array([0.0, 0.3, -1.2]) * ext, c, 50.0)[:npri]
    nd = n - npri
    rng = np.random.default_rng([seed, 3])
    k = rng.integers(0, v.shape[0], nd)
    u = rng.random((nd, 4), dtype=np.float32)
    su = np.sqrt(u[:, 0])
    w0, w1 = 1 - su, su * (1 - u[:, 1])
    w2 = su * u[:, 1]
    a, b, cc = v[k, 0], v[k, 1], v[k, 2]
    p = w0[:, None] * a + w1[:, None] * b + w2[:, None] * cc
    nrm = np.cross(b - a, cc - a)
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), F32(1e-30))
    t, bt = _onb(nrm)
    r, ph = np.sqrt(u[:, 2]), F32(2 * math.pi) * u[:, 3]
    x, y, z = r * np.cos(ph), r * np.sin(ph), np.sqrt(np.maximum(F32(0), 1 - u[:, 2]))
    d = x[:, None] * t + y[:, None] * bt + z[:, None] * nrm
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    dif = np.zeros(nd, dtype=RAY_DTYPE)
    dif["org"] = p + F32(1e-3) * ext * nrm
    dif["dir"] = d
    dif["tmin"] = 0.0
    dif["tmax"] = 1e30
    return np.concatenate([pri, dif])


# ----------------------------------------------------------- served trace --
def served_scenes(nscenes: int = 16, total: int = 30_000_000, lo: int = 200_000, hi: int = 5_000_000,
                  seed: int = 11, only=None):
    """Resident scenes of the served workload: sizes log-uniform in [lo, hi],
    rescaled so they sum to `total` (each kept within [lo, hi]); scene i =
    scene_meshes(seed=1000 + i, n_i), all in the same 100^3 box.  `only` (a
    range of scene ids, default all) makes just those scenes."""
    u = uniforms(seed, S_SERVE, nscenes, 4)[:, 0].astype(np.float64)
    w = log_uniform(u, lo, hi)
    n = np.clip(np.round(w * total / w.sum()), lo, hi).astype(int)
    n[-1] += total - n.sum()
    n = np.clip(n, lo, hi)
    with concurrent.futures.ThreadPoolExecutor(min(16, os.cpu_count() or 1)) as ex:
        return list(ex.map(lambda i: scene_meshes(1000 + i, int(n[i])), range(nscenes) if only is None else only))


def served_trace(nreq: int, rate: float = 2000.0, nscenes: int = 16, ray_lo: int = 1000, ray_hi: int = 8_000_000,
                 any_frac: float = 0.3, pool: int = 8_000_000, seed: int = 12):
    """Poisson request trace: arrival times (s, exponential gaps at `rate`),
    scene uniform, ray count log-uniform [ray_lo, ray_hi], any hit with
    probability any_frac, and the start of the request's window in a shared
    ray pool of `pool` rays."""
    u = uniforms(seed, S_SERVE + 1, nreq, 8).astype(np.float64)
    arrival = np.cumsum(-np.log1p(-u[:, 0]) / rate)
    arrival -= arrival[0]
    scene = np.minimum((u[:, 1] * nscenes).astype(int), nscenes - 1)
    n = np.round(log_uniform(u[:, 2], ray_lo, ray_hi)).astype(int)
    any_hit = u[:, 3] < any_frac
    start = np.floor(u[:, 4] * (pool - n + 1)).astype(int)
    return arrival, scene, n, any_hit, start


def served_ray_pools(n: int = 8_000_000, box: float = 100.0, seed: int = 13):
    """Shared pools for the served workload, drawn with numpy's PCG64 seeded
    by (seed, kind): incoherent closest-hit rays (uniform origins in the
    box, uniform directions) and any-hit segments of the same kind with
    length uniform in [10, 100]."""
    def pool(kind):
        rng = np.random.default_rng([seed, kind])
        u = rng.random((n, 6), dtype=np.float32)
        z = 2 * u[:, 3] - 1
        ph = F32(2 * math.pi) * u[:, 4]
        sr = np.sqrt(np.maximum(F32(0), 1 - z * z))
        r = np.zeros(n, dtype=RAY_DTYPE)
        r["org"] = (u[:, 0:3] - F32(0.5)) * F32(box)
        r["dir"] = np.stack([sr * np.cos(ph), sr * np.sin(ph), z], 1)
        r["tmin"] = 0.0
        r["tmax"] = 1e30 if kind == 0 else F32(10) + F32(90) * u[:, 5]
        return r
    return pool(0), pool(1)
