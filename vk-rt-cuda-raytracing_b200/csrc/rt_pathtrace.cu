// rt_pathtrace.cu -- wavefront path tracer over an instanced scene (the
// generate / extend / shade / shadow / finalize stages of cuda_rt_v34.cu:
// 1077-1497, re-specified for deterministic results).
//
// Per render: all W*H*spp paths are live at once (2M pixels x 8 spp = 16.6M
// path states, ~2 GB at 1080p x 8).  Each bounce launches
//   extend   two-level closest hit over the ray queue (rt_tlas.cu), count
//            read from device memory (no host round trip);
//   shade    one thread per queue entry: camera-hit emission, next-event
//            estimation toward one emissive triangle, cosine bounce, Russian
//            roulette; survivors and shadow rays are appended to their queues
//            with warp-ballot compaction (one atomic per warp);
//   shadow   two-level any hit over the shadow queue;
//   accum    unoccluded contributions added to the path's own radiance slot
//            (one writer per path per bounce, no atomics);
// then finalize averages the samples of each pixel in sample order.
//
// Model (fixed so the FP64 oracle can mirror it): Lambertian surfaces with
// per-instance albedo; emission counted only on camera hits; next-event
// estimation picks an emissive triangle with probability proportional to its
// world-space area, using an exact integer CDF (areas quantised to
// fixed point, 64-bit prefix sums), samples a uniform point on it; emitters
// are two-sided; black environment; Russian roulette from bounce rr_start with
// p = max(max component of throughput, 0.05).  Randomness: Philox4x32-10, key
// (seed, 0x50545201), counter (pixel, sample, bounce << 8 | purpose, 0).  All
// geometric quantities (rays, hit points, normals, light points, RR
// probability) use explicitly rounded fp32 operations, so the oracle's paths
// are the same paths; only radiance differs (fp32 here, fp64 there).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "rt_internal.h"
#include "rt_trace.cuh"

namespace rtb {

constexpr uint32_t PT_KEY = 0x50545201u;
constexpr float PT_EPS = 1e-3f;     // origin offset along the normal
constexpr float PT_TMIN = 1e-4f;
constexpr int PT_T = 256;
constexpr int kMaxBounces = 16;

struct PtScene {
    const float4* mat;        // 2 per instance: albedo, emission
    const float* fwd;         // 12 per instance
    const float* inv;         // 12 per instance
    const float* const* tris9;  // per instance: BLAS input triangles
    const unsigned long long* cdf;  // inclusive, per light triangle
    const int2* lights;       // (instance, primitive)
    int num_lights;
    unsigned long long total_q;
    float area_scale;         // total light area in world units^2
};

struct PtCam {
    float eye[3], f[3], r[3], u[3];
    float th, aspect;
};

__device__ __forceinline__ float dv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float sq(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return add(add(mul(ax, bx), mul(ay, by)), mul(az, bz));
}

__device__ __forceinline__ uint4 pt_rand(uint32_t pixel, uint32_t sample, uint32_t bounce, uint32_t purpose,
                                         uint32_t seed) {
    return philox(make_uint4(pixel, sample, (bounce << 8) | purpose, 0u), make_uint2(seed, PT_KEY));
}

// Warp-aggregated append: one atomicAdd per warp, ballot rank within it.
__device__ __forceinline__ int warp_append(bool want, int* counter) {
    const unsigned m = __ballot_sync(0xFFFFFFFFu, want);
    if (!m) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    return want ? base + __popc(m & ((1u << lane) - 1)) : -1;
}

// Camera paths p0 .. p0 + np - 1 (path = pixel * spp + sample) into queue
// slots 0 .. np - 1; throughput and radiance are indexed by path.
__global__ void k_pt_generate(PtCam c, int W, int H, int spp, uint32_t seed, int64_t p0, int np,
                              RtRay* __restrict__ rays, int* __restrict__ pid, float4* __restrict__ tp,
                              float4* __restrict__ L, int* __restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int64_t path = p0 + i;
    const uint32_t pixel = (uint32_t)(path / spp), s = (uint32_t)(path % spp);
    const uint32_t px = pixel % W, py = pixel / W;
    const uint4 rr = pt_rand(pixel, s, 0, 0, seed);
    const float j1 = u01(rr.x), j2 = u01(rr.y);
    const float x = mul(mul(sub(mul(dv(add((float)px, j1), (float)W), 2.f), 1.f), c.th), c.aspect);
    const float y = mul(sub(1.f, mul(dv(add((float)py, j2), (float)H), 2.f)), c.th);
    const float dx = add(add(c.f[0], mul(x, c.r[0])), mul(y, c.u[0]));
    const float dy = add(add(c.f[1], mul(x, c.r[1])), mul(y, c.u[1]));
    const float dz = add(add(c.f[2], mul(x, c.r[2])), mul(y, c.u[2]));
    const float len = sq(dot3(dx, dy, dz, dx, dy, dz));
    RtRay r;
    r.org[0] = c.eye[0]; r.org[1] = c.eye[1]; r.org[2] = c.eye[2]; r.tmin = 0.f;
    r.dir[0] = dv(dx, len); r.dir[1] = dv(dy, len); r.dir[2] = dv(dz, len); r.tmax = 1e30f;
    rays[i] = r;
    pid[i] = (int)path;
    tp[path] = make_float4(1.f, 1.f, 1.f, 0.f);
    L[path] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (i == 0) *count = np;
}

// Per-bounce ray counts of one slice added to the frame's totals.
__global__ void k_pt_count(const int* __restrict__ ext, const int* __restrict__ shadow, int* __restrict__ acc2) {
    acc2[0] += *ext;
    acc2[1] += *shadow;
}

// Shading waits on scattered loads (hit triangles, instances, lights): 6
// CTAs per SM (40 registers, some spilled) hide more of it than 4 at 64
// registers, +0.9 % on the frame; 8 (32 registers) +0.4 %.  The grid-stride
// launch is sized to exactly the resident CTAs (no ragged second wave:
// another +2.0 %).
#ifndef RTB_SHADE_MINB
#define RTB_SHADE_MINB 6
#endif
// RTB_SHADE_COMPACT: each warp lists the queue entries whose ray hit in
// shared memory and shades them 32 at a time, so no lane idles through a
// whole shade on a miss (a capture of one launch showed 13.5 of 32 lanes
// active).  Queue order changes, results do not: every path has its own
// radiance and throughput slot and its own random stream.
#ifndef RTB_SHADE_COMPACT
#define RTB_SHADE_COMPACT 1
#endif
__global__ void __launch_bounds__(PT_T, RTB_SHADE_MINB) k_pt_shade(PtScene sc, int spp, int bounce, int max_bounces, int rr_start,
                                                   uint32_t seed, const int* __restrict__ in_count,
                                                   const RtRay* __restrict__ rays, const int* __restrict__ pid,
                                                   const RtHit* __restrict__ hits, const int32_t* __restrict__ hinst,
                                                   float4* __restrict__ tp_arr, float4* __restrict__ L_arr,
                                                   RtRay* __restrict__ next_rays, int* __restrict__ next_pid,
                                                   int* __restrict__ next_count, RtRay* __restrict__ srays,
                                                   int* __restrict__ spid, float4* __restrict__ scontrib,
                                                   int* __restrict__ scount) {
    const int n = *in_count;
#if RTB_SHADE_COMPACT
    __shared__ int s_list[PT_T / 32][64];
    const int lane = threadIdx.x & 31;
    int* lst = s_list[threadIdx.x >> 5];
    int c = 0;  // entries listed; the same in every lane of the warp
    const int stride = gridDim.x * PT_T;
    int base = blockIdx.x * PT_T + (threadIdx.x & ~31);  // this warp's next 32 queue entries
    // whole warps stay in the loop so the ballots below see every lane
    for (;;) {
        while (c < 32 && base < n) {
            const int k = base + lane;
            const bool hit = k < n && hits[k].prim >= 0;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, hit);
            if (hit) lst[c + __popc(m & ((1u << lane) - 1))] = k;
            c += __popc(m);
            base += stride;
        }
        if (c == 0) break;
        const int take = c < 32 ? c : 32;
        __syncwarp();
        const int i = lane < take ? lst[lane] : 0;
        __syncwarp();
        if (lane < c - take) lst[lane] = lst[take + lane];  // the rest to the front (c - take < 32)
        c -= take;
        __syncwarp();
        bool live = lane < take;
#else
    // whole warps stay in the loop so the ballots below see every lane
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int i = base + threadIdx.x;
        bool live = i < n;
#endif
        RtHit h;
        int path = 0, inst = -1;
        if (live) {
            h = hits[i];
            path = pid[i];
            inst = hinst[i];
            live = h.prim >= 0;
        }
        bool want_shadow = false, want_next = false;
        RtRay sray, nray;
        float4 contrib = make_float4(0.f, 0.f, 0.f, 0.f);
        float4 tpn = make_float4(0.f, 0.f, 0.f, 0.f);
        if (live) {
            const RtRay r = rays[i];
            const uint32_t pixel = (uint32_t)(path / spp), s = (uint32_t)(path % spp);
            const float4 alb = sc.mat[2 * inst], emi = sc.mat[2 * inst + 1];
            const float4 tp = tp_arr[path];
            if (bounce == 0 && (emi.x > 0.f || emi.y > 0.f || emi.z > 0.f)) {
                float4 l = L_arr[path];
                l.x += tp.x * emi.x; l.y += tp.y * emi.y; l.z += tp.z * emi.z;
                L_arr[path] = l;
            }
            // hit point and world-space geometric normal facing the ray
            const float px = add(r.org[0], mul(h.t, r.dir[0]));
            const float py = add(r.org[1], mul(h.t, r.dir[1]));
            const float pz = add(r.org[2], mul(h.t, r.dir[2]));
            const float* tv = sc.tris9[inst] + (size_t)h.prim * 9;
            const float e1x = sub(tv[3], tv[0]), e1y = sub(tv[4], tv[1]), e1z = sub(tv[5], tv[2]);
            const float e2x = sub(tv[6], tv[0]), e2y = sub(tv[7], tv[1]), e2z = sub(tv[8], tv[2]);
            const float nox = sub(mul(e1y, e2z), mul(e1z, e2y));
            const float noy = sub(mul(e1z, e2x), mul(e1x, e2z));
            const float noz = sub(mul(e1x, e2y), mul(e1y, e2x));
            const float* iv = sc.inv + (size_t)inst * 12;
            float nx = add(add(mul(iv[0], nox), mul(iv[4], noy)), mul(iv[8], noz));
            float ny = add(add(mul(iv[1], nox), mul(iv[5], noy)), mul(iv[9], noz));
            float nz = add(add(mul(iv[2], nox), mul(iv[6], noy)), mul(iv[10], noz));
            const float nl = sq(dot3(nx, ny, nz, nx, ny, nz));
            nx = dv(nx, nl); ny = dv(ny, nl); nz = dv(nz, nl);
            if (dot3(nx, ny, nz, r.dir[0], r.dir[1], r.dir[2]) > 0.f) { nx = -nx; ny = -ny; nz = -nz; }
            const float ox = add(px, mul(PT_EPS, nx)), oy = add(py, mul(PT_EPS, ny)), oz = add(pz, mul(PT_EPS, nz));
            // next-event estimation
            if (sc.num_lights > 0) {
                const uint4 rl = pt_rand(pixel, s, bounce, 1, seed);
                const unsigned long long r64 = ((unsigned long long)rl.x << 32) | rl.y;
                const unsigned long long target = __umul64hi(r64, sc.total_q);
                int lo = 0, hi = sc.num_lights - 1;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (sc.cdf[mid] > target) hi = mid;
                    else lo = mid + 1;
                }
                const int2 lt = sc.lights[lo];
                const float* lv = sc.tris9[lt.x] + (size_t)lt.y * 9;
                const float* fw = sc.fwd + (size_t)lt.x * 12;
                float ax, ay, az, bx, by, bz, cx, cy, cz;
                xform_point(fw, lv[0], lv[1], lv[2], ax, ay, az);
                xform_point(fw, lv[3], lv[4], lv[5], bx, by, bz);
                xform_point(fw, lv[6], lv[7], lv[8], cx, cy, cz);
                const float su = sq(u01(rl.z)), xb = u01(rl.w);
                const float wa = sub(1.f, su), wb = mul(su, sub(1.f, xb)), wc = mul(su, xb);
                const float lx = add(add(mul(wa, ax), mul(wb, bx)), mul(wc, cx));
                const float ly = add(add(mul(wa, ay), mul(wb, by)), mul(wc, cy));
                const float lz = add(add(mul(wa, az), mul(wb, bz)), mul(wc, cz));
                const float f1x = sub(bx, ax), f1y = sub(by, ay), f1z = sub(bz, az);
                const float f2x = sub(cx, ax), f2y = sub(cy, ay), f2z = sub(cz, az);
                const float gx = sub(mul(f1y, f2z), mul(f1z, f2y));
                const float gy = sub(mul(f1z, f2x), mul(f1x, f2z));
                const float gz = sub(mul(f1x, f2y), mul(f1y, f2x));
                const float gl = sq(dot3(gx, gy, gz, gx, gy, gz));
                const float tx = sub(lx, ox), ty = sub(ly, oy), tz = sub(lz, oz);
                const float d2 = dot3(tx, ty, tz, tx, ty, tz);
                const float dist = sq(d2);
                if (dist > 0.f && gl > 0.f) {
                    const float dx = dv(tx, dist), dy = dv(ty, dist), dz = dv(tz, dist);
                    const float cx_ = dot3(nx, ny, nz, dx, dy, dz);
                    const float cl = dv(fabsf(dot3(gx, gy, gz, dx, dy, dz)), gl);
                    if (cx_ > 0.f && cl > 0.f) {
                        const float4 le = sc.mat[2 * lt.x + 1];
                        const float gterm = cx_ * cl / d2 * sc.area_scale * 0.3183098861837907f;
                        contrib = make_float4(tp.x * alb.x * le.x * gterm, tp.y * alb.y * le.y * gterm,
                                              tp.z * alb.z * le.z * gterm, 0.f);
                        sray.org[0] = ox; sray.org[1] = oy; sray.org[2] = oz; sray.tmin = PT_TMIN;
                        sray.dir[0] = dx; sray.dir[1] = dy; sray.dir[2] = dz; sray.tmax = mul(dist, 0.9999f);
                        want_shadow = true;
                    }
                }
            }
            // continuation: cosine-weighted bounce (Malley on a rejection-sampled disk)
            if (bounce + 1 < max_bounces) {
                float tx, ty, tz;
                if (fabsf(nx) > fabsf(ny)) {
                    const float il = dv(1.f, sq(add(mul(nx, nx), mul(nz, nz))));
                    tx = -mul(nz, il); ty = 0.f; tz = mul(nx, il);
                } else {
                    const float il = dv(1.f, sq(add(mul(ny, ny), mul(nz, nz))));
                    tx = 0.f; ty = mul(nz, il); tz = -mul(ny, il);
                }
                const float bx = sub(mul(ny, tz), mul(nz, ty));
                const float by = sub(mul(nz, tx), mul(nx, tz));
                const float bz = sub(mul(nx, ty), mul(ny, tx));
                float x = 0.f, y = 0.f;
                bool got = false;
                for (int q = 0; q < 4 && !got; q++) {
                    const uint4 rd = pt_rand(pixel, s, bounce, 3 + q, seed);
                    const uint32_t w4[4] = {rd.x, rd.y, rd.z, rd.w};
                    for (int k = 0; k < 2 && !got; k++) {
                        const float a = sub(mul(u01(w4[2 * k]), 2.f), 1.f);
                        const float b = sub(mul(u01(w4[2 * k + 1]), 2.f), 1.f);
                        if (add(mul(a, a), mul(b, b)) < 1.f) { x = a; y = b; got = true; }
                    }
                }
                const float z = sq(fmaxf(0.f, sub(sub(1.f, mul(x, x)), mul(y, y))));
                float dx = add(add(mul(x, tx), mul(y, bx)), mul(z, nx));
                float dy = add(add(mul(x, ty), mul(y, by)), mul(z, ny));
                float dz = add(add(mul(x, tz), mul(y, bz)), mul(z, nz));
                const float dl = sq(dot3(dx, dy, dz, dx, dy, dz));
                dx = dv(dx, dl); dy = dv(dy, dl); dz = dv(dz, dl);
                float t0 = mul(tp.x, alb.x), t1 = mul(tp.y, alb.y), t2 = mul(tp.z, alb.z);
                bool cont = true;
                if (bounce >= rr_start) {
                    const float p = fmaxf(fmaxf(fmaxf(t0, t1), t2), 0.05f);
                    const float xi = u01(pt_rand(pixel, s, bounce, 2, seed).x);
                    if (xi >= p) cont = false;
                    else { t0 = dv(t0, p); t1 = dv(t1, p); t2 = dv(t2, p); }
                }
                if (cont) {
                    nray.org[0] = ox; nray.org[1] = oy; nray.org[2] = oz; nray.tmin = PT_TMIN;
                    nray.dir[0] = dx; nray.dir[1] = dy; nray.dir[2] = dz; nray.tmax = 1e30f;
                    tpn = make_float4(t0, t1, t2, 0.f);
                    want_next = true;
                }
            }
        }
        const int si = warp_append(want_shadow, scount);
        if (want_shadow) {
            srays[si] = sray;
            spid[si] = path;
            scontrib[si] = contrib;
        }
        const int ni = warp_append(want_next, next_count);
        if (want_next) {
            next_rays[ni] = nray;
            next_pid[ni] = path;
            tp_arr[path] = tpn;
        }
    }
}

__global__ void k_pt_accum(const int* __restrict__ count, const int* __restrict__ spid,
                           const float4* __restrict__ contrib, const uint8_t* __restrict__ occ,
                           float4* __restrict__ L_arr) {
    const int n = *count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (occ[i]) continue;
        const int p = spid[i];
        const float4 c = contrib[i];
        float4 l = L_arr[p];
        l.x += c.x; l.y += c.y; l.z += c.z;
        L_arr[p] = l;
    }
}

__global__ void k_pt_finalize(const float4* __restrict__ L_arr, int pixels, int spp, float* __restrict__ rgb) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    if (px >= pixels) return;
    float r = 0.f, g = 0.f, b = 0.f;
    for (int s = 0; s < spp; s++) {
        const float4 l = L_arr[(size_t)px * spp + s];
        r += l.x; g += l.y; b += l.z;
    }
    const float k = 1.f / (float)spp;
    rgb[(size_t)px * 3 + 0] = r * k;
    rgb[(size_t)px * 3 + 1] = g * k;
    rgb[(size_t)px * 3 + 2] = b * k;
}

__global__ void k_zero2(int* a, int* b) {
    *a = 0;
    *b = 0;
}

}  // namespace rtb

using namespace rtb;

struct RtPathTracerHandle {
    CudaTLAS_t tlas = nullptr;
    unsigned long long tlas_generation = 0;  // the TLAS's instances this tracer copied
    int ninst = 0;
    std::vector<char> emissive;                  // per instance
    std::vector<std::vector<float>> host_tris;   // per BLAS, emissive ones only (light table)
    DevBuf<float4> mat;
    DevBuf<float> fwd, inv;
    DevBuf<const float*> tris9;
    DevBuf<unsigned long long> cdf;
    DevBuf<int2> lights;
    int num_lights = 0;
    unsigned long long total_q = 0;
    double light_area = 0.0;
    // per-render buffers: queues for `cap` paths (a slice of the frame), per-path
    // throughput and radiance for `cap_paths` (the whole frame)
    int64_t cap = 0, cap_paths = 0;
    int64_t queue_paths = 0;  // rtPT_setQueueCapacity: paths per slice, 0 = the whole frame
    DevBuf<RtRay> rays[2], srays;
    DevBuf<int> pid[2], spid, counts;
    DevBuf<RtHit> hits;
    DevBuf<int32_t> hinst;
    DevBuf<float4> tp, L, scontrib;
    DevBuf<uint8_t> socc;
    DevBuf<int> work;
    unsigned work_next = 0;
    DevBuf<int> bcounts;      // per bounce: extension rays, shadow rays
    RtPTStats stats{};
    // extension-queue regrouping (rtPT_setRegroup): key kind and bits (0 = off),
    // the world box the origin Morton codes are taken in, sorted queue copies
    int regroup_kind = RT_REGROUP_OCTANT_MORTON, regroup_bits = 0;
    float world_box[6] = {0, 0, 0, 0, 0, 0};
    DevBuf<RtRay> rays_sorted;
    DevBuf<int> pid_sorted;
};

namespace {

// Host camera basis (double, then fp32) shared with the oracle through
// rtPT_cameraBasis.
PtCam make_cam(const RtCamera& c, int W, int H) {
    double f[3], r[3], u[3];
    for (int a = 0; a < 3; a++) f[a] = (double)c.target[a] - (double)c.eye[a];
    double fl = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (int a = 0; a < 3; a++) f[a] /= fl;
    r[0] = f[1] * c.up[2] - f[2] * c.up[1];
    r[1] = f[2] * c.up[0] - f[0] * c.up[2];
    r[2] = f[0] * c.up[1] - f[1] * c.up[0];
    double rl = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (int a = 0; a < 3; a++) r[a] /= rl;
    u[0] = r[1] * f[2] - r[2] * f[1];
    u[1] = r[2] * f[0] - r[0] * f[2];
    u[2] = r[0] * f[1] - r[1] * f[0];
    PtCam pc;
    for (int a = 0; a < 3; a++) {
        pc.eye[a] = c.eye[a];
        pc.f[a] = (float)f[a];
        pc.r[a] = (float)r[a];
        pc.u[a] = (float)u[a];
    }
    pc.th = (float)tan(c.vfov_deg * 3.14159265358979323846 / 360.0);
    pc.aspect = (float)((double)W / (double)H);
    return pc;
}

// World area of an instance triangle, double, fixed operation order
// (mirrored by the oracle).
double tri_area_world(const float* m, const float* v) {
    double p[3][3];
    for (int k = 0; k < 3; k++)
        for (int r = 0; r < 3; r++)
            p[k][r] = (double)m[r * 4] * v[k * 3] + (double)m[r * 4 + 1] * v[k * 3 + 1] +
                      (double)m[r * 4 + 2] * v[k * 3 + 2] + (double)m[r * 4 + 3];
    const double a[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    const double b[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    const double c[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    return 0.5 * sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
}

}  // namespace

// Instance-dependent state of a tracer, from the transforms (12 floats per
// instance) and BLAS choices given: forward / inverse transforms, each
// instance's BLAS triangles, and the emissive triangles weighted by world
// area (an exact integer CDF).  Host copies of emissive BLASes are kept for
// later reloads.
// World box of the TLAS (its binary root), for the regrouping keys.
static bool load_world_box(RtPathTracerHandle* pt) {
    Node2 root;
    if (!RT_CUDA(cudaMemcpy(&root, pt->tlas->bvh2.nodes.p, sizeof(Node2), cudaMemcpyDeviceToHost))) return false;
    for (int a = 0; a < 3; a++) {
        pt->world_box[a] = root.lo[a];
        pt->world_box[3 + a] = root.hi[a];
    }
    return true;
}

static bool load_instances(RtPathTracerHandle* pt, const float* fwd12, const int* blas_idx, const char* who) {
    const CudaTLASHandle* tlas = pt->tlas;
    const int ni = pt->ninst;
    std::vector<const float*> t9(ni);
    std::vector<double> areas;
    std::vector<int2> lights;
    for (int k = 0; k < ni; k++) {
        const int b = blas_idx[k];
        if (b < 0 || b >= (int)tlas->blas.size()) {
            set_error("%s: instance %d names BLAS %d", who, k, b);
            return false;
        }
        const CudaBVHHandle* bh = tlas->blas[b];
        t9[k] = bh->tris9.p;
        if (pt->emissive[k]) {
            std::vector<float>& ht = pt->host_tris[b];
            if (ht.empty()) {
                ht.resize((size_t)bh->num_tris * 9);
                if (!RT_CUDA(cudaMemcpy(ht.data(), bh->tris9.p, ht.size() * 4, cudaMemcpyDeviceToHost))) return false;
            }
            for (int p = 0; p < bh->num_tris; p++) {
                areas.push_back(tri_area_world(fwd12 + (size_t)12 * k, &ht[(size_t)p * 9]));
                lights.push_back(make_int2(k, p));
            }
        }
    }
    pt->total_q = 0;
    pt->light_area = 0.0;
    // exact integer CDF: q_i = floor(area_i * 2^K), K from count and max area
    pt->num_lights = (int)lights.size();
    std::vector<unsigned long long> cdf(lights.size());
    if (!lights.empty()) {
        double amax = 0.0;
        for (double a : areas) amax = std::max(amax, a);
        const int K = (int)floor(61.0 - log2((double)areas.size() * std::max(amax, 1e-300)));
        unsigned long long run = 0;
        for (size_t i = 0; i < areas.size(); i++) {
            run += (unsigned long long)floor(ldexp(areas[i], K));
            cdf[i] = run;
        }
        pt->total_q = run;
        pt->light_area = ldexp((double)run, -K);
    }
    const size_t nl = std::max<size_t>(lights.size(), 1);
    bool ok = pt->fwd.ensure((size_t)12 * ni) && pt->inv.ensure((size_t)12 * ni) && pt->tris9.ensure(ni) &&
              pt->cdf.ensure(nl) && pt->lights.ensure(nl) &&
              RT_CUDA(cudaMemcpy(pt->fwd.p, fwd12, (size_t)12 * ni * 4, cudaMemcpyHostToDevice)) &&
              RT_CUDA(cudaMemcpy(pt->inv.p, tlas->h_inv.data(), (size_t)12 * ni * 4, cudaMemcpyHostToDevice)) &&
              RT_CUDA(cudaMemcpy(pt->tris9.p, t9.data(), t9.size() * sizeof(void*), cudaMemcpyHostToDevice));
    if (ok && !lights.empty())
        ok = RT_CUDA(cudaMemcpy(pt->cdf.p, cdf.data(), cdf.size() * 8, cudaMemcpyHostToDevice)) &&
             RT_CUDA(cudaMemcpy(pt->lights.p, lights.data(), lights.size() * 8, cudaMemcpyHostToDevice));
    if (!ok) return false;
    pt->stats.light_tris = pt->num_lights;
    pt->stats.light_area = pt->light_area;
    return true;
}

extern "C" {

int rtPT_cameraBasis(const RtCamera* cam, int width, int height, float* out14) {
    if (!cam || width <= 0 || height <= 0 || !out14) {
        set_error("rtPT_cameraBasis: invalid argument");
        return RT_ERR_INVALID;
    }
    const PtCam c = make_cam(*cam, width, height);
    memcpy(out14, &c, sizeof(float) * 14);
    return RT_OK;
}

RtPathTracer_t rtPT_create(CudaTLAS_t tlas, const RtMaterial* mats, int nmat, const RtInstance* instances) {
    clear_error();
    if (!tlas || !mats || !instances || nmat != tlas->num_instances) {
        set_error("rtPT_create: need one material and one instance record per TLAS instance");
        return nullptr;
    }
    RtPathTracerHandle* pt = new (std::nothrow) RtPathTracerHandle();
    if (!pt) return nullptr;
    pt->tlas = tlas;
    pt->tlas_generation = tlas->generation;
    const int ni = nmat;
    pt->ninst = ni;
    std::vector<float4> mat((size_t)2 * ni);
    std::vector<float> fwd((size_t)12 * ni);
    std::vector<int> bidx(ni);
    pt->emissive.assign(ni, 0);
    pt->host_tris.assign(tlas->blas.size(), std::vector<float>());
    for (int k = 0; k < ni; k++) {
        mat[2 * k] = make_float4(mats[k].albedo[0], mats[k].albedo[1], mats[k].albedo[2], 0.f);
        mat[2 * k + 1] = make_float4(mats[k].emission[0], mats[k].emission[1], mats[k].emission[2], 0.f);
        memcpy(&fwd[(size_t)12 * k], instances[k].xform, 48);
        bidx[k] = instances[k].blas;
        pt->emissive[k] = mats[k].emission[0] > 0.f || mats[k].emission[1] > 0.f || mats[k].emission[2] > 0.f;
    }
    bool ok = pt->mat.alloc(mat.size()) && pt->counts.alloc(8) && pt->work.alloc(1024) &&
              pt->bcounts.alloc(2 * kMaxBounces) &&
              RT_CUDA(cudaMemcpy(pt->mat.p, mat.data(), mat.size() * 16, cudaMemcpyHostToDevice)) &&
              load_instances(pt, fwd.data(), bidx.data(), "rtPT_create") && load_world_box(pt);
    if (!ok) {
        delete pt;
        return nullptr;
    }
    return pt;
}

int rtPT_setQueueCapacity(RtPathTracer_t pt, int64_t paths) {
    if (!pt || paths < 0) {
        set_error("rtPT_setQueueCapacity: invalid argument");
        return RT_ERR_INVALID;
    }
    pt->queue_paths = paths;
    return RT_OK;
}

int rtPT_autotune(RtPathTracer_t pt, const RtCamera* cam, const RtPTParams* prm, float* d_rgb, void* stream,
                  int64_t* out_paths) {
    if (!pt || !cam || !prm || !d_rgb || prm->width <= 0 || prm->height <= 0 || prm->spp <= 0) {
        set_error("rtPT_autotune: invalid argument");
        return RT_ERR_INVALID;
    }
    const int64_t P = (int64_t)prm->width * prm->height * prm->spp;
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!RT_CUDA(cudaEventCreate(&e0)) || !RT_CUDA(cudaEventCreate(&e1))) return RT_ERR_CUDA;
    int64_t best_q = 0;
    float best = 1e30f;
    int rc = RT_OK;
    // the whole frame, then slices of 1/2, 1/4 and 1/8 of it (whole pixels)
    for (int div : {1, 2, 4, 8}) {
        const int64_t q = div == 1 ? 0 : ((P / div + prm->spp - 1) / prm->spp) * prm->spp;
        if (div > 1 && q < (int64_t)num_sms() * 4096) break;  // too small a slice to fill the GPU
        pt->queue_paths = q;
        if ((rc = rtPT_render(pt, cam, prm, d_rgb, stream)) != RT_OK) break;  // warm (allocates)
        if (!RT_CUDA(cudaEventRecord(e0, s))) { rc = RT_ERR_CUDA; break; }
        if ((rc = rtPT_render(pt, cam, prm, d_rgb, stream)) != RT_OK) break;
        float ms = 0.f;
        if (!RT_CUDA(cudaEventRecord(e1, s)) || !RT_CUDA(cudaEventSynchronize(e1)) ||
            !RT_CUDA(cudaEventElapsedTime(&ms, e0, e1))) {
            rc = RT_ERR_CUDA;
            break;
        }
        if (ms < best) {
            best = ms;
            best_q = q;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    pt->queue_paths = best_q;
    if (out_paths) *out_paths = best_q;
    return rc;
}

int rtPT_setRegroup(RtPathTracer_t pt, int kind, int key_bits) {
    if (!pt || (key_bits != 0 && key_bits != 16 && key_bits != 32) ||
        (kind != RT_REGROUP_MORTON && kind != RT_REGROUP_OCTANT_MORTON)) {
        set_error("rtPT_setRegroup: invalid argument");
        return RT_ERR_INVALID;
    }
    pt->regroup_kind = kind;
    pt->regroup_bits = key_bits;
    return RT_OK;
}

void rtPT_destroy(RtPathTracer_t pt) {
    if (!pt) return;
    cudaDeviceSynchronize();
    delete pt;
}

int rtPT_render(RtPathTracer_t pt, const RtCamera* cam, const RtPTParams* prm, float* d_rgb, void* stream) {
    if (!pt || !cam || !prm || !d_rgb || prm->width <= 0 || prm->height <= 0 || prm->spp <= 0 ||
        prm->max_bounces <= 0 || prm->max_bounces > kMaxBounces) {
        set_error("rtPT_render: invalid argument");
        return RT_ERR_INVALID;
    }
    if (misaligned(d_rgb, 4)) {
        set_error("rtPT_render: d_rgb must be 4-byte aligned");
        return RT_ERR_INVALID;
    }
    // The TLAS lock is held from the reload check to the last launch, so a
    // cudaTLAS_setTransforms on another thread cannot swap the instances or
    // the top level between this render's launches.
    std::lock_guard<std::mutex> tlas_lock(pt->tlas->mu);
    // the TLAS's instances moved (cudaTLAS_setTransforms): reload the copies
    // once renders still in flight are done with them
    if (pt->tlas->generation != pt->tlas_generation) {
        const CudaTLASHandle* t = pt->tlas;
        if (!RT_CUDA(cudaDeviceSynchronize()) || !load_instances(pt, t->h_fwd.data(), t->h_blas.data(), "rtPT_render") ||
            !load_world_box(pt))
            return RT_ERR_CUDA;
        pt->tlas_generation = t->generation;
    }
    const int64_t P = (int64_t)prm->width * prm->height * prm->spp;
    if (P > (int64_t)INT32_MAX) {
        set_error("rtPT_render: %lld paths exceed 2^31", (long long)P);
        return RT_ERR_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    // queues hold one slice of Q paths; the frame is traced slice after slice
    const int64_t Q = pt->queue_paths > 0 ? std::min(pt->queue_paths, P) : P;
    if (P > pt->cap_paths) {
        if (!pt->tp.alloc(P) || !pt->L.alloc(P)) return RT_ERR_NOMEM;
        pt->cap_paths = P;
    }
    if (Q > pt->cap) {
        const bool ok = pt->rays[0].alloc(Q) && pt->rays[1].alloc(Q) && pt->srays.alloc(Q) && pt->pid[0].alloc(Q) &&
                        pt->pid[1].alloc(Q) && pt->spid.alloc(Q) && pt->hits.alloc(Q) && pt->hinst.alloc(Q) &&
                        pt->scontrib.alloc(Q) && pt->socc.alloc(Q);
        if (!ok) return RT_ERR_NOMEM;
        pt->cap = Q;
        pt->rays_sorted.release();
        pt->pid_sorted.release();
    }
    if (pt->regroup_bits && (!pt->rays_sorted.ensure(pt->cap) || !pt->pid_sorted.ensure(pt->cap))) return RT_ERR_NOMEM;
    CudaTLASHandle* t = pt->tlas;
    PtScene sc;
    sc.mat = pt->mat.p;
    sc.fwd = pt->fwd.p;
    sc.inv = pt->inv.p;
    sc.tris9 = pt->tris9.p;
    sc.cdf = pt->cdf.p;
    sc.lights = pt->lights.p;
    sc.num_lights = pt->num_lights;
    sc.total_q = pt->total_q;
    sc.area_scale = (float)pt->light_area;
    const PtCam c = make_cam(*cam, prm->width, prm->height);
    int* cnt = pt->counts.p;  // [0],[1]: ray queues, [2]: shadow queue
    cudaMemsetAsync(pt->bcounts.p, 0, sizeof(int) * 2 * kMaxBounces, s);
    const int shade_blocks = num_sms() * 8;
    for (int64_t p0 = 0; p0 < P; p0 += Q) {
        const int np = (int)std::min(Q, P - p0);
        k_pt_generate<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(c, prm->width, prm->height, prm->spp, prm->seed, p0,
                                                                  np, pt->rays[0].p, pt->pid[0].p, pt->tp.p, pt->L.p, cnt);
        int cur = 0;
        for (int b = 0; b < prm->max_bounces; b++) {
            const int nxt = cur ^ 1;
            k_zero2<<<1, 1, 0, s>>>(cnt + nxt, cnt + 2);
            int* w1 = pt->work.p + (pt->work_next++ % 1024);
            cudaMemsetAsync(w1, 0, sizeof(int), s);
            // bounce rays leave scattered surface points in all directions: regroup
            // them (direction octant, origin Morton code) before the extension trace;
            // camera rays (bounce 0) are already in pixel order
            RtRay* qrays = pt->rays[cur].p;
            int* qpid = pt->pid[cur].p;
            if (pt->regroup_bits && b > 0) {
                if (!regroup_rays(qrays, qpid, (int)pt->cap, cnt + cur, 0, pt->world_box, pt->regroup_kind,
                                  pt->regroup_bits, pt->rays_sorted.p, pt->pid_sorted.p, nullptr, s))
                    return RT_ERR_CUDA;
                qrays = pt->rays_sorted.p;
                qpid = pt->pid_sorted.p;
            }
            if (launch_trace_tlas(t, qrays, 0, cnt + cur, pt->hits.p, pt->hinst.p, nullptr, w1, t->status.p, s) != RT_OK)
                return RT_ERR_CUDA;
            k_pt_shade<<<num_sms() * RTB_SHADE_MINB, PT_T, 0, s>>>(sc, prm->spp, b, prm->max_bounces, prm->rr_start, prm->seed,
                                                     cnt + cur, qrays, qpid, pt->hits.p,
                                                     pt->hinst.p, pt->tp.p, pt->L.p, pt->rays[nxt].p, pt->pid[nxt].p,
                                                     cnt + nxt, pt->srays.p, pt->spid.p, pt->scontrib.p, cnt + 2);
            int* w2 = pt->work.p + (pt->work_next++ % 1024);
            cudaMemsetAsync(w2, 0, sizeof(int), s);
            if (launch_trace_tlas(t, pt->srays.p, 0, cnt + 2, nullptr, nullptr, pt->socc.p, w2, t->status.p, s) != RT_OK)
                return RT_ERR_CUDA;
            k_pt_accum<<<shade_blocks, 256, 0, s>>>(cnt + 2, pt->spid.p, pt->scontrib.p, pt->socc.p, pt->L.p);
            // ray counts of this bounce for the statistics
            k_pt_count<<<1, 1, 0, s>>>(cnt + cur, cnt + 2, pt->bcounts.p + 2 * b);
            cur = nxt;
        }
    }  // slices
    const int pixels = prm->width * prm->height;
    k_pt_finalize<<<(pixels + 255) / 256, 256, 0, s>>>(pt->L.p, pixels, prm->spp, d_rgb);
    return RT_CUDA(cudaGetLastError()) ? RT_OK : RT_ERR_CUDA;
}

int rtPT_getStats(RtPathTracer_t pt, RtPTStats* out) {
    if (!pt || !out) {
        set_error("rtPT_getStats: invalid argument");
        return RT_ERR_INVALID;
    }
    int bc[2 * kMaxBounces];
    if (!RT_CUDA(cudaMemcpy(bc, pt->bcounts.p, sizeof(bc), cudaMemcpyDeviceToHost))) return RT_ERR_CUDA;
    RtPTStats s = pt->stats;
    s.extension_rays = 0;
    s.shadow_rays = 0;
    for (int b = 0; b < kMaxBounces; b++) {
        s.extension_rays += (uint64_t)bc[b * 2];
        s.shadow_rays += (uint64_t)bc[b * 2 + 1];
    }
    *out = s;
    return RT_OK;
}

}  // extern "C"
