// rt_tlas.cu -- TLAS over instanced BLASes: GPU build and two-level
// closest/any-hit traversal (the two-level walk of layer/rt_ir_exec.cu:93-189
// and the instance records of layer/VkLayer_CudaRT.cpp:4517-4558, done on
// the compressed 8-wide layout).
//
// Build: world box of every instance = the bounds of its BLAS's vertices
// under its transform (evaluated on the GPU in double precision, rounded
// outward to float), padded outward by a relative 2^-16 of the coordinate
// magnitudes (covers the rounding of the object-space ray transform), then
// the same GPU SAH builder with one instance per leaf.
// Trace: one stack for both levels.  Entering an instance transforms the
// world ray by the inverse 3x4 (no renormalisation, t stays in world units)
// and switches node/triangle arrays; node groups pushed at the top level
// carry a flag, so popping one restores the world ray.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "rt_internal.h"
#include "rt_trace.cuh"

namespace rtb {

constexpr uint32_t G_TOP = 1u << 16;   // group belongs to the top level
constexpr uint32_t G_INST = 1u << 17;  // group is a mask of instance leaves
constexpr int INST_F4 = 6;             // float4 words per instance record

// Instance record (6 x float4): inverse 3x4 rows, BLAS node and triangle
// pointers, the instance's base in the global (instance, primitive)
// numbering used for tie breaks, and the object-space bounds of the BLAS's
// vertices (base, lo.xyz), (hi.xyz, 0).
struct InstView {
    float m[12];
    const uint4* nodes;
    const float4* tris;
    uint32_t base;
    float lo[3], hi[3];
};

__device__ __forceinline__ InstView load_inst(const float4* __restrict__ inst, int i) {
    const float4* ip = inst + (size_t)i * INST_F4;
    const float4 r0 = __ldg(ip), r1 = __ldg(ip + 1), r2 = __ldg(ip + 2), pp = __ldg(ip + 3), bb = __ldg(ip + 4),
                 bh = __ldg(ip + 5);
    InstView v;
    v.m[0] = r0.x; v.m[1] = r0.y; v.m[2] = r0.z; v.m[3] = r0.w;
    v.m[4] = r1.x; v.m[5] = r1.y; v.m[6] = r1.z; v.m[7] = r1.w;
    v.m[8] = r2.x; v.m[9] = r2.y; v.m[10] = r2.z; v.m[11] = r2.w;
    v.nodes = reinterpret_cast<const uint4*>(((unsigned long long)__float_as_uint(pp.y) << 32) | __float_as_uint(pp.x));
    v.tris = reinterpret_cast<const float4*>(((unsigned long long)__float_as_uint(pp.w) << 32) | __float_as_uint(pp.z));
    v.base = __float_as_uint(bb.x);
    v.lo[0] = bb.y; v.lo[1] = bb.z; v.lo[2] = bb.w;
    v.hi[0] = bh.x; v.hi[1] = bh.y; v.hi[2] = bh.z;
    return v;
}

// Whether the object-space ray can meet the box within [tmin, thit]: the
// slab distances (p - o) / d carry a relative slack of 2^-22 and the far
// distance one of 2^-21, which bound the roundings of the subtraction, the
// product and the guarded reciprocal, so a box holding an accepted hit is
// never culled (the node test's argument, with the planes given directly).
__device__ __forceinline__ bool box_reached(const Ray& r, const float (&lo)[3], const float (&hi)[3], float tmin,
                                           float thit) {
    const float ax = (lo[0] - r.ox) * r.ix, bx = (hi[0] - r.ox) * r.ix;
    const float ay = (lo[1] - r.oy) * r.iy, by = (hi[1] - r.oy) * r.iy;
    const float az = (lo[2] - r.oz) * r.iz, bz = (hi[2] - r.oz) * r.iz;
    const float nx = fminf(ax, bx), fx = fmaxf(ax, bx);
    const float ny = fminf(ay, by), fy = fmaxf(ay, by);
    const float nz = fminf(az, bz), fz = fmaxf(az, bz);
    const float tn = max3f(fmaf(-fabsf(nx), 0x1p-22f, nx), fmaf(-fabsf(ny), 0x1p-22f, ny),
                           fmaxf(fmaf(-fabsf(nz), 0x1p-22f, nz), tmin));
    const float tf = min3f(fmaf(fabsf(fx), 0x1p-22f, fx), fmaf(fabsf(fy), 0x1p-22f, fy),
                           fminf(fmaf(fabsf(fz), 0x1p-22f, fz), thit));
    return tn <= fmaf(fabsf(tf), 0x1p-21f, tf);
}

// Two-level closest/any hit.  Same iteration structure as the single-level
// kernel (rt_trace.cu): up to RTB_NODE_ITERS steps per lane (a step visits a
// top or bottom node, or enters the next instance of an instance group),
// then the warp-pooled triangle phase over the lanes walking a BLAS; the
// shared key's low word is the global id base(instance) + primitive, so one
// 64-bit atomicMin resolves ties by (t, instance, primitive).
// Closest hit keeps more state across the two levels than the single-level
// kernel: 7 CTAs per SM (72 registers) measured +0.8 % on the path tracer
// over 8 (64 registers, more spilled); any hit stays at 8.
#ifndef RTB_TLAS_MINB
#define RTB_TLAS_MINB 7
#endif
// Steps per lane per iteration of this kernel (a step is a node visit or
// entering an instance) and its node test's slot-mask mode (RTB_SLOTMASK in
// rt_trace.cuh), tuned apart from the single-level kernel on the path
// tracer (1080p x 8 spp, 5M triangles): 2 steps 1,323 Mrays/s, 3: 1,393,
// 4: 1,466, 6: 1,503; with the meta-byte table (mode 2) 3: 1,425, 4: 1,495,
// 6: 1,527.
#ifndef RTB_TLAS_ITERS
#define RTB_TLAS_ITERS 6
#endif
#ifndef RTB_TLAS_SLOTMASK
#define RTB_TLAS_SLOTMASK 2
#endif
// RTB_TLAS_PACK: plane distances by packed f32x2 FMAs (RTB_PACK_CLOSEST in
// rt_trace.cuh), closest and any hit: path tracer +1.7 % (1,751 -> 1,780
// Mrays/s, image identical).
#ifndef RTB_TLAS_PACK
#define RTB_TLAS_PACK 1
#endif
// RTB_TLAS_SMEM: a lane entering an instance also writes its instance-space
// ray and its instance (triangle array, id base, index) to shared memory,
// where the lanes testing its triangles read them (three 16-byte loads)
// instead of gathering them with thirteen shuffles per pooled round.
#ifndef RTB_TLAS_SMEM
#define RTB_TLAS_SMEM 1
#endif
// RTB_TLAS_TWO_SETS (with RTB_TLAS_SMEM): a lane keeps two pending sets of
// leaf triangles, each with its own instance (ray, triangle array, id base)
// written to shared memory when the set is recorded, so a step that finds
// leaves does not end the lane's steps and the second set may come from
// another instance.
#ifndef RTB_TLAS_TWO_SETS
#define RTB_TLAS_TWO_SETS 0
#endif
// RTB_TLAS_STATS (analysis builds only; the release kernel is unchanged):
// event counters in g_tlas_stats, read by rtTlasStats_read: [0] warp
// iterations, [1] lanes holding a ray at an iteration's start, [2] instance
// entries, [3] top-level node visits, [4] bottom-level node visits,
// [5] triangle tests, [6] 32-lane triangle rounds, [7] rays finished,
// [8] instances skipped by their object-space box.
#ifndef RTB_TLAS_STATS
#define RTB_TLAS_STATS 0
#endif
// RTB_TLAS_ROOTBOX: after transforming the ray into an instance, test the
// object-space bounds of its BLAS (an oriented box in world space, tighter
// than the instance's world-axis box for a rotated instance) before
// visiting the BLAS's root node.
#ifndef RTB_TLAS_ROOTBOX
#define RTB_TLAS_ROOTBOX 1
#endif
#if RTB_TLAS_STATS
__device__ unsigned long long g_tlas_stats[9];
#endif

template <bool ANY>
__global__ void __launch_bounds__(TRACE_T, ANY ? TRACE_MINB : RTB_TLAS_MINB)
    k_trace_tlas(const uint4* __restrict__ tnodes, const int* __restrict__ leaf_ids, const float4* __restrict__ inst,
                 const RtRay* __restrict__ rays, int n, const int* __restrict__ n_dev, RtHit* __restrict__ hits,
                 int32_t* __restrict__ inst_out, uint8_t* __restrict__ occ, int* __restrict__ work,
                 int* __restrict__ status) {
    __shared__ uint2 sstack[SSTACK][TRACE_T];
    __shared__ unsigned long long s_key[TRACE_T];
    __shared__ int s_rec[TRACE_T];
    __shared__ int4 s_res[TRACE_T];  // u, v bits, instance, primitive of the improved best
#if RTB_TLAS_SMEM
    constexpr int NSET = RTB_TLAS_TWO_SETS ? 2 : 1;
    __shared__ float4 s_ray[NSET][2][TRACE_T];  // per pending set: instance-space ray (o, world tmin), (d, world tmax)
    __shared__ uint4 s_inst[NSET][TRACE_T];     // per pending set: triangle array (lo, hi), id base, instance index
#endif
    static_assert(!RTB_TLAS_TWO_SETS || RTB_TLAS_SMEM, "two pending sets keep their instances in shared memory");
#if RTB_TLAS_SLOTMASK
    __shared__ NodeLuts s_luts;
    init_node_luts(&s_luts);
    const NodeLuts* s_oct_perm = &s_luts;
#else
    const NodeLuts* s_oct_perm = nullptr;
#endif
    if (n_dev) n = *n_dev;  // ray count produced on the device by an earlier stage
    uint2 lstack[LSTACK];
    const int lane = threadIdx.x & 31;
    const int wbase = threadIdx.x & ~31;
    int ray = -1;
    bool exhausted = false;
    Ray wr, cr;
    Walk w;
    bool in_blas = false;
    const uint4* bnodes = nullptr;
    const float4* btris = nullptr;
    int cur_inst = -1;
    uint32_t cur_base = 0;
    float thit = 0.f, hu = 0.f, hv = 0.f;
    int hprim = -1, hinst = -1;
    uint32_t hid = 0xFFFFFFFFu;
#if RTB_TLAS_STATS
    unsigned long long st_entry = 0, st_top = 0, st_bot = 0, st_done = 0, st_skip = 0;
#endif
    for (;;) {
        const bool need = ray < 0 && !exhausted;
        const unsigned want = __ballot_sync(FULL_MASK, need);
        if (want) {
            const int leader = __ffs(want) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(work, __popc(want));
            base = __shfl_sync(FULL_MASK, base, leader);
            if (need) {
                const int ri = base + __popc(want & ((1u << lane) - 1));
                if (ri < n) {
                    ray = ri;
                    wr = load_ray(rays, ri);
                    cr = wr;
                    in_blas = false;
                    thit = wr.tmax;
                    hprim = hinst = -1;
                    hid = 0xFFFFFFFFu;
                    hu = hv = 0.f;
                    w.start();
                    w.ng = make_uint2(0u, (1u << wr.oct) | (1u << 8) | G_TOP);
                } else {
                    exhausted = true;
                }
            }
        }
        if (__all_sync(FULL_MASK, ray < 0)) break;
#if RTB_TLAS_STATS
        {
            const unsigned hold = __ballot_sync(FULL_MASK, ray >= 0);
            if (lane == 0) {
                atomicAdd(&g_tlas_stats[0], 1ull);
                atomicAdd(&g_tlas_stats[1], (unsigned long long)__popc(hold));
            }
        }
#endif
        // ---- node phase ----
        uint32_t tri_base = 0, tmask = 0;
#if RTB_TLAS_TWO_SETS
        uint32_t tri_base2 = 0, tmask2 = 0;  // a second set while the first waits
#define RTB_TLAS_LAST tmask2
#else
        constexpr uint32_t tmask2 = 0;
#define RTB_TLAS_LAST tmask
#endif
        bool overflow = false;
#pragma unroll 1
        for (int it = 0; it < RTB_TLAS_ITERS; it++) {
            if (ray < 0 || RTB_TLAS_LAST || overflow) break;
            if (w.ng.y & G_INST) {
                // enter the next instance of an instance group
                uint32_t m = w.ng.y & 0xFFu;
                const int j = __ffs(m) - 1;
                m &= m - 1;
                const int next_inst = leaf_ids[w.ng.x + j];
                const InstView iv = load_inst(inst, next_inst);
                float ox, oy, oz, dx, dy, dz;
                xform_point(iv.m, wr.ox, wr.oy, wr.oz, ox, oy, oz);
                xform_dir(iv.m, wr.dx, wr.dy, wr.dz, dx, dy, dz);
                const Ray tr = make_ray(make_float4(ox, oy, oz, wr.tmin), make_float4(dx, dy, dz, wr.tmax));
#if RTB_TLAS_ROOTBOX
                if (!box_reached(tr, iv.lo, iv.hi, wr.tmin, thit)) {
                    // the instance's own box is missed: its root node is not visited;
                    // the group's other instances (or the next stacked group) come next
#if RTB_TLAS_STATS
                    st_skip++;
#endif
                    if (m) {
                        w.ng.y = (w.ng.y & ~0xFFu) | m;
                    } else {
                        w.ng.y = 0;
                        if (w.sp > 0) w.ng = w.pop(sstack, lstack);  // at the top level: the world ray stays
                    }
                    continue;
                }
#endif
                if (m && !w.push(make_uint2(w.ng.x, m | G_INST | G_TOP), sstack, lstack)) {
                    overflow = true;
                    break;
                }
                cur_inst = next_inst;
#if RTB_TLAS_STATS
                st_entry++;
#endif
                cr = tr;
                bnodes = iv.nodes;
                btris = iv.tris;
                cur_base = iv.base;
                in_blas = true;
#if RTB_TLAS_SMEM && !RTB_TLAS_TWO_SETS
                s_ray[0][0][threadIdx.x] = make_float4(cr.ox, cr.oy, cr.oz, wr.tmin);
                s_ray[0][1][threadIdx.x] = make_float4(cr.dx, cr.dy, cr.dz, wr.tmax);
                s_inst[0][threadIdx.x] = make_uint4((uint32_t)(unsigned long long)btris,
                                                    (uint32_t)((unsigned long long)btris >> 32), cur_base,
                                                    (uint32_t)cur_inst);
#endif
                w.ng = make_uint2(0u, (1u << cr.oct) | (1u << 8));
                continue;
            }
            if ((w.ng.y & 0xFFu) == 0) break;
            uint32_t hitsm = w.ng.y & 0xFFu;
            const uint32_t imask = (w.ng.y >> 8) & 0xFFu;
            const uint32_t top = w.ng.y & G_TOP;
            const int k = __ffs(hitsm) - 1;
            hitsm &= hitsm - 1;
            const uint32_t slot = (uint32_t)k ^ cr.oct;
            const uint32_t ni = w.ng.x + __popc(imask & ((1u << slot) - 1));
            if (hitsm && !w.push(make_uint2(w.ng.x, hitsm | (imask << 8) | top), sstack, lstack)) {
                overflow = true;
                break;
            }
            uint32_t nh, tb, tm;
#if RTB_TLAS_STATS
            if (top) st_top++;
            else st_bot++;
#endif
            visit_node<RTB_TLAS_SLOTMASK, RTB_TLAS_PACK != 0>((top ? tnodes : bnodes) + (size_t)ni * 5, cr, thit, nh, tb, tm, w.ng,
                                          s_oct_perm);
            if (top) {
                w.ng.y |= G_TOP;
                if (tm) {
                    // instance leaves: keep the node group, walk the instances next
                    if ((w.ng.y & 0xFFu) && !w.push(w.ng, sstack, lstack)) {
                        overflow = true;
                        break;
                    }
                    w.ng = make_uint2(tb, (tm & 0xFFu) | G_INST | G_TOP);
                }
            } else {
#if RTB_TLAS_TWO_SETS
                if (tm) {
                    const int set = tmask ? 1 : 0;
                    if (set) {
                        tri_base2 = tb;
                        tmask2 = tm;
                    } else {
                        tri_base = tb;
                        tmask = tm;
                    }
                    s_ray[set][0][threadIdx.x] = make_float4(cr.ox, cr.oy, cr.oz, wr.tmin);
                    s_ray[set][1][threadIdx.x] = make_float4(cr.dx, cr.dy, cr.dz, wr.tmax);
                    s_inst[set][threadIdx.x] = make_uint4((uint32_t)(unsigned long long)btris,
                                                          (uint32_t)((unsigned long long)btris >> 32), cur_base,
                                                          (uint32_t)cur_inst);
                }
#else
                tri_base = tb;
                tmask = tm;
#endif
            }
            if ((w.ng.y & 0xFFu) == 0 && !(w.ng.y & G_INST) && (RTB_TLAS_TWO_SETS || !tmask) && w.sp > 0) {
                w.ng = w.pop(sstack, lstack);
                if (in_blas && (w.ng.y & G_TOP)) {
                    in_blas = false;
                    cr = wr;
                }
            }
        }
#undef RTB_TLAS_LAST
        // ---- triangle phase: pooled over the warp ----
        const int cnt = __popc(tmask) + __popc(tmask2);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL_MASK, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(FULL_MASK, incl, 31);
#if RTB_TLAS_STATS
        if (lane == 0 && total) {
            atomicAdd(&g_tlas_stats[5], (unsigned long long)total);
            atomicAdd(&g_tlas_stats[6], (unsigned long long)((total + 31) / 32));
        }
#endif
        bool found_any = false;
        if (total) {
            const int excl = incl - cnt;
            if (!ANY) s_key[threadIdx.x] = ((unsigned long long)f2ord(thit) << 32) | hid;
            s_rec[threadIdx.x] = ANY ? 0 : -1;
            __syncwarp();
#if !RTB_TLAS_SMEM
            const unsigned long long tp64 = (unsigned long long)btris;
#endif
            for (int b = 0; b < total; b += 32) {
                const int g = b + lane;
                int o = 0;
#pragma unroll
                for (int s = 16; s; s >>= 1) {
                    const int v = __shfl_sync(FULL_MASK, incl, o + s - 1);
                    if (v <= g) o += s;
                }
                o = min(o, 31);
                const int k0 = g - __shfl_sync(FULL_MASK, excl, o);
                uint32_t om = __shfl_sync(FULL_MASK, tmask, o);
                uint32_t ob = __shfl_sync(FULL_MASK, tri_base, o);
#if RTB_TLAS_TWO_SETS
                const uint32_t om2 = __shfl_sync(FULL_MASK, tmask2, o);
                const uint32_t ob2 = __shfl_sync(FULL_MASK, tri_base2, o);
                const int c1 = __popc(om);
                const int set = k0 >= c1 ? 1 : 0;
                const int k = set ? k0 - c1 : k0;
                if (set) {
                    om = om2;
                    ob = ob2;
                }
#else
                constexpr int set = 0;
                const int k = k0;
#endif
#if RTB_TLAS_SMEM
                const uint4 oi = s_inst[set][wbase + o];
                const unsigned long long optr = ((unsigned long long)oi.y << 32) | oi.x;
                const uint32_t obase = oi.z;
                const int oinst = (int)oi.w;
                const float4 ro = s_ray[set][0][wbase + o], rd = s_ray[set][1][wbase + o];
                const float ox = ro.x, oy = ro.y, oz = ro.z, tmn = ro.w;
                const float dx = rd.x, dy = rd.y, dz = rd.z, tmx = rd.w;
#else
                const unsigned long long optr = __shfl_sync(FULL_MASK, tp64, o);
                const uint32_t obase = __shfl_sync(FULL_MASK, cur_base, o);
                const int oinst = __shfl_sync(FULL_MASK, cur_inst, o);
                const float ox = __shfl_sync(FULL_MASK, cr.ox, o), oy = __shfl_sync(FULL_MASK, cr.oy, o),
                            oz = __shfl_sync(FULL_MASK, cr.oz, o);
                const float dx = __shfl_sync(FULL_MASK, cr.dx, o), dy = __shfl_sync(FULL_MASK, cr.dy, o),
                            dz = __shfl_sync(FULL_MASK, cr.dz, o);
                const float tmn = __shfl_sync(FULL_MASK, wr.tmin, o), tmx = __shfl_sync(FULL_MASK, wr.tmax, o);
#endif
                unsigned long long key = ~0ull;
                float u = 0.f, v = 0.f;
                int prim = 0;
                if (g < total) {
                    const int rec = (int)ob + (int)nth_set_bit(om, (uint32_t)k);
                    const float4* tp = reinterpret_cast<const float4*>(optr) + (size_t)rec * 3;
                    const float4 A = __ldg(tp), B = __ldg(tp + 1), Cc = __ldg(tp + 2);
                    float t;
                    if (intersect_tri(ox, oy, oz, dx, dy, dz, A, B, Cc, t, u, v) && t > tmn && t < tmx) {
                        prim = __float_as_int(A.w);
                        if (ANY) s_rec[wbase + o] = 1;
                        else key = ((unsigned long long)f2ord(t) << 32) | (obase + (uint32_t)prim);
                    }
                }
                if (!ANY) {
                    if (key != ~0ull) atomicMin(&s_key[wbase + o], key);
                    __syncwarp();
                    if (key != ~0ull && s_key[wbase + o] == key) {
                        s_rec[wbase + o] = 1;
                        s_res[wbase + o] = make_int4(__float_as_int(u), __float_as_int(v), oinst, prim);
                    }
                    __syncwarp();
                }
            }
            __syncwarp();
            if (ANY) {
                found_any = s_rec[threadIdx.x] != 0;
            } else if (s_rec[threadIdx.x] >= 0) {
                const unsigned long long key = s_key[threadIdx.x];
                const int4 res = s_res[threadIdx.x];
                thit = ord2f((uint32_t)(key >> 32));
                hid = (uint32_t)key;
                hu = __int_as_float(res.x);
                hv = __int_as_float(res.y);
                hinst = res.z;
                hprim = res.w;
            }
        }
        // ---- advance / finish ----
        if (ray >= 0) {
            bool done = overflow || (ANY && found_any);
            if (!done && (w.ng.y & 0xFFu) == 0 && !(w.ng.y & G_INST)) {
                if (w.sp == 0) {
                    done = true;
                } else {
                    w.ng = w.pop(sstack, lstack);
                    if (in_blas && (w.ng.y & G_TOP)) {
                        in_blas = false;
                        cr = wr;
                    }
                }
            }
            if (done) {
                if (overflow) {
                    atomicOr(status, RT_STATUS_STACK);
                    hprim = -1;
                    found_any = false;
                }
                if (ANY) {
                    occ[ray] = found_any ? 1 : 0;
                } else {
                    reinterpret_cast<float4*>(hits)[ray] =
                        make_float4(hprim >= 0 ? thit : __int_as_float(0x7f800000), __int_as_float(hprim),
                                    hprim >= 0 ? hu : 0.f, hprim >= 0 ? hv : 0.f);
                    if (inst_out) inst_out[ray] = hprim >= 0 ? hinst : -1;
                }
#if RTB_TLAS_STATS
                st_done++;
#endif
                ray = -1;
            }
        }
    }
#if RTB_TLAS_STATS
    atomicAdd(&g_tlas_stats[2], st_entry);
    atomicAdd(&g_tlas_stats[3], st_top);
    atomicAdd(&g_tlas_stats[4], st_bot);
    atomicAdd(&g_tlas_stats[7], st_done);
    atomicAdd(&g_tlas_stats[8], st_skip);
#endif
}

#if RTB_TLAS_STATS
extern "C" int rtTlasStats_read(unsigned long long* out9, int reset) {
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpyFromSymbol(out9, g_tlas_stats, sizeof(unsigned long long) * 9) != cudaSuccess)
        return -1;
    if (reset) {
        static const unsigned long long zero[9] = {};
        if (cudaMemcpyToSymbol(g_tlas_stats, zero, sizeof(zero)) != cudaSuccess) return -1;
    }
    return 0;
}
#endif

template <class K>
static int grid_for(K kernel) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, TRACE_T, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    return per_sm * num_sms();
}

int launch_trace_tlas(const CudaTLASHandle* t, const RtRay* rays, int n, const int* n_dev, RtHit* hits,
                      int32_t* inst_out, uint8_t* occ, int* work, int* status, cudaStream_t s) {
    const uint4* nodes = reinterpret_cast<const uint4*>(t->bvh8.nodes.p);
    if (occ) {
        static const int g = grid_for(k_trace_tlas<true>);
        k_trace_tlas<true><<<g, TRACE_T, 0, s>>>(nodes, t->bvh8.leaf_ids.p, t->inst.p, rays, n, n_dev, hits,
                                                 inst_out, occ, work, status);
    } else {
        static const int g = grid_for(k_trace_tlas<false>);
        k_trace_tlas<false><<<g, TRACE_T, 0, s>>>(nodes, t->bvh8.leaf_ids.p, t->inst.p, rays, n, n_dev, hits,
                                                  inst_out, occ, work, status);
    }
    return RT_CUDA(cudaGetLastError()) ? RT_OK : RT_ERR_CUDA;
}

static float bits_f(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// inverse of a row-major affine 3x4 in double
static bool invert34(const float* m, double* inv) {
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
    const double A = e * i - f * h, B = -(d * i - f * g), Cc = d * h - e * g;
    const double det = a * A + b * B + c * Cc;
    if (!(fabs(det) > 1e-300)) return false;
    const double id = 1.0 / det;
    double r[9] = {A * id, -(b * i - c * h) * id, (b * f - c * e) * id,
                   B * id, (a * i - c * g) * id, -(a * f - c * d) * id,
                   Cc * id, -(a * h - b * g) * id, (a * e - b * d) * id};
    const double tx = m[3], ty = m[7], tz = m[11];
    for (int row = 0; row < 3; row++) {
        inv[row * 4 + 0] = r[row * 3 + 0];
        inv[row * 4 + 1] = r[row * 3 + 1];
        inv[row * 4 + 2] = r[row * 3 + 2];
        inv[row * 4 + 3] = -(r[row * 3 + 0] * tx + r[row * 3 + 1] * ty + r[row * 3 + 2] * tz);
    }
    return true;
}

// World bounds of the instances' geometry: the BLAS's vertices under the
// instance's transform, one CTA row per instance (grid.y), sums of exact
// float products in double, min / max rounded outward to float and folded
// into ordered-uint atomics (6 per instance: lo xyz, hi xyz).  Tighter than
// the transformed corners of the BLAS's root box, which for a rotated
// instance bound a box around a box: fewer rays enter an instance they then
// miss (the path tracer's scene: 72 % of the surface area of the corner
// boxes), and hits do not change (the boxes still hold every triangle).
struct InstBoundsJob {
    const float* tris9;  // the BLAS's input triangles, 9 floats each
    int ntris;
    float m[12];         // object -> world, row-major 3x4
};

__global__ void k_instance_bounds(const InstBoundsJob* __restrict__ jobs, uint32_t* __restrict__ out) {
    const InstBoundsJob j = jobs[blockIdx.y];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    float olo[3] = {INFINITY, INFINITY, INFINITY}, ohi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const int nv = j.ntris * 3;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
        const float* v = j.tris9 + (size_t)i * 3;
        const double x = v[0], y = v[1], z = v[2];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            olo[r] = fminf(olo[r], v[r]);
            ohi[r] = fmaxf(ohi[r], v[r]);
        }
#pragma unroll
        for (int r = 0; r < 3; r++) {
            const double w = (double)j.m[r * 4] * x + (double)j.m[r * 4 + 1] * y + (double)j.m[r * 4 + 2] * z +
                             (double)j.m[r * 4 + 3];
            lo[r] = fmin(lo[r], w);
            hi[r] = fmax(hi[r], w);
        }
    }
#pragma unroll
    for (int r = 0; r < 3; r++) {
        for (int o = 16; o; o >>= 1) {
            lo[r] = fmin(lo[r], __shfl_xor_sync(FULL_MASK, lo[r], o));
            hi[r] = fmax(hi[r], __shfl_xor_sync(FULL_MASK, hi[r], o));
            olo[r] = fminf(olo[r], __shfl_xor_sync(FULL_MASK, olo[r], o));
            ohi[r] = fmaxf(ohi[r], __shfl_xor_sync(FULL_MASK, ohi[r], o));
        }
    }
    if ((threadIdx.x & 31) == 0 && nv > 0) {
        uint32_t* o12 = out + (size_t)blockIdx.y * 12;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            atomicMin(&o12[r], f2ord(__double2float_rd(lo[r])));
            atomicMax(&o12[3 + r], f2ord(__double2float_ru(hi[r])));
            atomicMin(&o12[6 + r], f2ord(olo[r]));
            atomicMax(&o12[9 + r], f2ord(ohi[r]));
        }
    }
}

// The instances' world bounds (see k_instance_bounds), padded outward by
// 2^-16 of the box's coordinate magnitude plus its extents, as float4 lo/hi.
static bool instance_bounds(const std::vector<CudaBVH_t>& blas, const RtInstance* inst, int ni,
                            std::vector<float4>& lo, std::vector<float4>& hi, std::vector<float>& obj6) {
    std::vector<InstBoundsJob> jobs(ni);
    int maxtris = 0;
    for (int k = 0; k < ni; k++) {
        const CudaBVHHandle* b = blas[inst[k].blas];
        if (!b->tris9.p || b->num_tris <= 0) {
            set_error("TLAS: BLAS %d holds no triangles", inst[k].blas);
            return false;
        }
        jobs[k].tris9 = b->tris9.p;
        jobs[k].ntris = b->num_tris;
        memcpy(jobs[k].m, inst[k].xform, sizeof(jobs[k].m));
        maxtris = std::max(maxtris, b->num_tris);
    }
    std::vector<uint32_t> h((size_t)ni * 12);
    for (int k = 0; k < ni; k++)
        for (int r = 0; r < 12; r++) h[(size_t)k * 12 + r] = (r < 3 || (r >= 6 && r < 9)) ? 0xFFFFFFFFu : 0u;
    DevBuf<InstBoundsJob> d_jobs;
    DevBuf<uint32_t> d_out;
    if (!d_jobs.alloc(ni) || !d_out.alloc((size_t)ni * 12) ||
        !RT_CUDA(cudaMemcpy(d_jobs.p, jobs.data(), sizeof(InstBoundsJob) * ni, cudaMemcpyHostToDevice)) ||
        !RT_CUDA(cudaMemcpy(d_out.p, h.data(), sizeof(uint32_t) * h.size(), cudaMemcpyHostToDevice)))
        return false;
    const int gx = std::max(1, std::min((3 * maxtris + 255) / 256, 64));
    if (ni > 65535) {
        set_error("TLAS: %d instances, at most 65535", ni);
        return false;
    }
    k_instance_bounds<<<dim3(gx, ni), 256>>>(d_jobs.p, d_out.p);
    if (!RT_CUDA(cudaGetLastError()) ||
        !RT_CUDA(cudaMemcpy(h.data(), d_out.p, sizeof(uint32_t) * h.size(), cudaMemcpyDeviceToHost)))
        return false;
    lo.resize(ni);
    hi.resize(ni);
    obj6.resize((size_t)ni * 6);
    auto ordf = [](uint32_t u) {
        const uint32_t v = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
        float f;
        memcpy(&f, &v, 4);
        return (double)f;
    };
    for (int k = 0; k < ni; k++) {
        double wl[3], wh[3], mag = 0.0;
        double ol[3], oh[3], omag = 0.0;
        for (int r = 0; r < 3; r++) {
            wl[r] = ordf(h[(size_t)k * 12 + r]);
            wh[r] = ordf(h[(size_t)k * 12 + 3 + r]);
            mag = std::max(mag, std::max(fabs(wl[r]), fabs(wh[r])));
            ol[r] = ordf(h[(size_t)k * 12 + 6 + r]);
            oh[r] = ordf(h[(size_t)k * 12 + 9 + r]);
            omag = std::max(omag, std::max(fabs(ol[r]), fabs(oh[r])));
        }
        // the object-space box gets the world box's relative pad: the kernels
        // test v0 + fl(v1 - v0) and v0 + fl(v2 - v0), which can lie a rounding
        // outside the input vertices' bounds, and the triangle test accepts
        // rays grazing an edge within its own rounding
        const double opad = ldexp(omag + (oh[0] - ol[0]) + (oh[1] - ol[1]) + (oh[2] - ol[2]), -16);
        for (int r = 0; r < 3; r++) {
            obj6[(size_t)k * 6 + r] = nextafterf((float)(ol[r] - opad), -INFINITY);
            obj6[(size_t)k * 6 + 3 + r] = nextafterf((float)(oh[r] + opad), INFINITY);
        }
        const double pad = ldexp(mag + (wh[0] - wl[0]) + (wh[1] - wl[1]) + (wh[2] - wl[2]), -16);
        lo[k] = make_float4(nextafterf((float)(wl[0] - pad), -INFINITY), nextafterf((float)(wl[1] - pad), -INFINITY),
                            nextafterf((float)(wl[2] - pad), -INFINITY), 0.f);
        hi[k] = make_float4(nextafterf((float)(wh[0] + pad), INFINITY), nextafterf((float)(wh[1] + pad), INFINITY),
                            nextafterf((float)(wh[2] + pad), INFINITY), 0.f);
    }
    return true;
}

// Per instance: the inverse transform (12 floats), the record the kernels
// read (inverse as 3 float4, BLAS node / record pointers, tie-break id
// base) and the padded world box of its geometry.  False, with the error
// set, on a bad instance.
static bool instance_data(const std::vector<CudaBVH_t>& blas, const RtInstance* inst, int ni, const char* who,
                          std::vector<float>& h_inv, std::vector<float4>& rec, std::vector<float4>& lo,
                          std::vector<float4>& hi) {
    const int nb = (int)blas.size();
    h_inv.assign((size_t)ni * 12, 0.f);
    rec.assign((size_t)ni * INST_F4, make_float4(0.f, 0.f, 0.f, 0.f));
    unsigned long long id_base = 0;
    for (int k = 0; k < ni; k++) {
        const RtInstance& I = inst[k];
        if (I.blas < 0 || I.blas >= nb) {
            set_error("%s: instance %d names BLAS %d of %d", who, k, I.blas, nb);
            return false;
        }
        double inv[12];
        if (!invert34(I.xform, inv)) {
            set_error("%s: instance %d transform is singular", who, k);
            return false;
        }
        float* fi = &h_inv[(size_t)k * 12];
        for (int j = 0; j < 12; j++) fi[j] = (float)inv[j];
        const CudaBVHHandle* b = blas[I.blas];
        const unsigned long long np = (unsigned long long)b->bvh8.nodes.p, tp = (unsigned long long)b->bvh8.tris.p;
        rec[(size_t)k * INST_F4 + 0] = make_float4(fi[0], fi[1], fi[2], fi[3]);
        rec[(size_t)k * INST_F4 + 1] = make_float4(fi[4], fi[5], fi[6], fi[7]);
        rec[(size_t)k * INST_F4 + 2] = make_float4(fi[8], fi[9], fi[10], fi[11]);
        rec[(size_t)k * INST_F4 + 4] = make_float4(bits_f((uint32_t)id_base), 0.f, 0.f, 0.f);
        id_base += (unsigned long long)b->num_tris;
        rec[(size_t)k * INST_F4 + 3] = make_float4(bits_f((uint32_t)np), bits_f((uint32_t)(np >> 32)), bits_f((uint32_t)tp),
                                             bits_f((uint32_t)(tp >> 32)));
    }
    if (id_base >= 0xFFFFFFFFull) {
        set_error("%s: %llu instance primitives exceed the 32-bit tie-break id", who, id_base);
        return false;
    }
    std::vector<float> obj6;
    if (!instance_bounds(blas, inst, ni, lo, hi, obj6)) return false;
    for (int k = 0; k < ni; k++) {
        const float* o = &obj6[(size_t)k * 6];
        float4& w4 = rec[(size_t)k * INST_F4 + 4];
        w4.y = o[0];
        w4.z = o[1];
        w4.w = o[2];
        rec[(size_t)k * INST_F4 + 5] = make_float4(o[3], o[4], o[5], 0.f);
    }
    return true;
}

// The instances as given: transform (12 floats) and BLAS index each.
static void instance_copy(const RtInstance* inst, int ni, std::vector<float>& fwd, std::vector<int>& blas) {
    fwd.resize((size_t)ni * 12);
    blas.resize(ni);
    for (int k = 0; k < ni; k++) {
        memcpy(&fwd[(size_t)k * 12], inst[k].xform, 12 * sizeof(float));
        blas[k] = inst[k].blas;
    }
}

// The top-level tree over the instance boxes: binned SAH with leaves of one
// instance, collapsed greedily to 8-wide nodes.
static bool build_top(const std::vector<float4>& lo, const std::vector<float4>& hi, Bvh2Device& b2, Bvh8Device& b8) {
    const int ni = (int)lo.size();
    DevBuf<float4> dlo, dhi;
    BuildConfig cfg;
    cfg.max_leaf = 1;
    return dlo.alloc(ni) && dhi.alloc(ni) &&
           RT_CUDA(cudaMemcpy(dlo.p, lo.data(), ni * sizeof(float4), cudaMemcpyHostToDevice)) &&
           RT_CUDA(cudaMemcpy(dhi.p, hi.data(), ni * sizeof(float4), cudaMemcpyHostToDevice)) &&
           build_bvh2(dlo.p, dhi.p, ni, cfg, b2, 0) && collapse_bvh8(b2, nullptr, b8, 0) &&
           RT_CUDA(cudaDeviceSynchronize()) &&
           (!getenv("RTB200_VALIDATE") || !atoi(getenv("RTB200_VALIDATE")) ||
            validate_bvh8(b8, b8.num_leaf_items, ni));
}

}  // namespace rtb

using namespace rtb;

extern "C" {

CudaTLAS_t cudaTLAS_build(const CudaBVH_t* blas, int nb, const RtInstance* inst, int ni) {
    clear_error();
    if (!blas || nb <= 0 || !inst || ni <= 0) {
        set_error("cudaTLAS_build: empty input");
        return nullptr;
    }
    for (int i = 0; i < nb; i++)
        if (!blas[i]) {
            set_error("cudaTLAS_build: BLAS %d is NULL", i);
            return nullptr;
        }
    CudaTLASHandle* t = new (std::nothrow) CudaTLASHandle();
    if (!t) return nullptr;
    t->num_instances = ni;
    t->blas.assign(blas, blas + nb);
    std::vector<float4> rec, lo, hi;
    instance_copy(inst, ni, t->h_fwd, t->h_blas);
    bool ok = instance_data(t->blas, inst, ni, "cudaTLAS_build", t->h_inv, rec, lo, hi) &&
              t->inst.alloc(rec.size()) &&
              RT_CUDA(cudaMemcpy(t->inst.p, rec.data(), rec.size() * sizeof(float4), cudaMemcpyHostToDevice)) &&
              build_top(lo, hi, t->bvh2, t->bvh8) && ensure_counters(t->counters) && t->status.alloc(1) &&
              RT_CUDA(cudaMemset(t->status.p, 0, sizeof(int))) && RT_CUDA(cudaDeviceSynchronize());
    if (!ok) {
        delete t;
        return nullptr;
    }
    return t;
}

// Per-frame instance update (the layer's processPendingTLAS,
// layer/VkLayer_CudaRT.cpp:3418, rebuilds its TLAS every CUDA_RT_TLAS_EVERY_N
// frames): new transforms and BLAS choices for the same number of
// instances, the top-level tree rebuilt in place; the BLASes are untouched.
// A path tracer on the TLAS reloads the instances at its next render.
int cudaTLAS_setTransforms(CudaTLAS_t t, const RtInstance* inst, int ni) {
    clear_error();
    if (!t || !inst || ni != t->num_instances) {
        set_error("cudaTLAS_setTransforms: need one instance record per TLAS instance (%d)",
                  t ? t->num_instances : 0);
        return RT_ERR_INVALID;
    }
    std::lock_guard<std::mutex> g(t->mu);
    std::vector<float> h_inv;
    std::vector<float4> rec, lo, hi;
    if (!instance_data(t->blas, inst, ni, "cudaTLAS_setTransforms", h_inv, rec, lo, hi)) return RT_ERR_INVALID;
    // the new tree is built aside, so a failure leaves the TLAS as it was
    Bvh2Device b2;
    Bvh8Device b8;
    if (!build_top(lo, hi, b2, b8)) return RT_ERR_CUDA;
    // traces still in flight read the current arrays: let them finish
    if (!RT_CUDA(cudaDeviceSynchronize()) ||
        !RT_CUDA(cudaMemcpy(t->inst.p, rec.data(), rec.size() * sizeof(float4), cudaMemcpyHostToDevice)))
        return RT_ERR_CUDA;
    t->bvh2.swap(b2);
    t->bvh8.swap(b8);
    t->h_inv.swap(h_inv);
    instance_copy(inst, ni, t->h_fwd, t->h_blas);
    t->generation++;
    return RT_OK;
}

void cudaTLAS_destroy(CudaTLAS_t t) {
    if (!t) return;
    cudaDeviceSynchronize();
    delete t;
}

int cudaTLAS_traceClosest(CudaTLAS_t t, const RtRay* d_rays, int n, RtHit* d_hits, int32_t* d_inst, void* stream) {
    if (!t || n < 0 || (n > 0 && (!d_rays || !d_hits))) {
        set_error("cudaTLAS_traceClosest: invalid argument");
        return RT_ERR_INVALID;
    }
    if (!check_aligned("cudaTLAS_traceClosest", d_rays, d_hits, 16)) return RT_ERR_INVALID;
    if (misaligned(d_inst, 4)) {
        set_error("cudaTLAS_traceClosest: d_inst must be 4-byte aligned");
        return RT_ERR_INVALID;
    }
    if (n == 0) return RT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    std::lock_guard<std::mutex> g(t->mu);  // not while cudaTLAS_setTransforms swaps the instances
    int* work = next_counter(t->counters, t->counter_next, s);
    return launch_trace_tlas(t, d_rays, n, nullptr, d_hits, d_inst, nullptr, work, t->status.p, s);
}

int cudaTLAS_traceAny(CudaTLAS_t t, const RtRay* d_rays, int n, uint8_t* d_occ, void* stream) {
    if (!t || n < 0 || (n > 0 && (!d_rays || !d_occ))) {
        set_error("cudaTLAS_traceAny: invalid argument");
        return RT_ERR_INVALID;
    }
    if (!check_aligned("cudaTLAS_traceAny", d_rays, d_occ, 1)) return RT_ERR_INVALID;
    if (n == 0) return RT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    std::lock_guard<std::mutex> g(t->mu);
    int* work = next_counter(t->counters, t->counter_next, s);
    return launch_trace_tlas(t, d_rays, n, nullptr, nullptr, nullptr, d_occ, work, t->status.p, s);
}

int cudaTLAS_getStatus(CudaTLAS_t t, void* stream) {
    if (!t) {
        set_error("cudaTLAS_getStatus: invalid argument");
        return RT_ERR_INVALID;
    }
    return read_status(t->status.p, (cudaStream_t)stream, "cudaTLAS_getStatus");
}

int cudaTLAS_getInverseTransforms(CudaTLAS_t t, float* out, int n) {
    if (!t || !out || n != t->num_instances) {
        set_error("cudaTLAS_getInverseTransforms: invalid argument");
        return RT_ERR_INVALID;
    }
    memcpy(out, t->h_inv.data(), t->h_inv.size() * sizeof(float));
    return RT_OK;
}

}  // extern "C"
