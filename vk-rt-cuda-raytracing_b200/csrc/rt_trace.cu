// rt_trace.cu -- closest-hit and any-hit traversal of the compressed 8-wide
// BVH (replaces bk_tracePrimaryDense / bk_traceDiffuseArbitrary,
// layer/cuda_bvh_backend.cu:104-183,526-598, and the any-hit traceShadow,
// v10_pipeline.cu:195-251).
//
// Execution model (B200, 148 SMs): persistent warps sized to fill every SM;
// each lane owns one ray; idle lanes refill from a global ray counter with
// one warp-aggregated atomic (dynamic fetch), so warps stay full while ray
// lengths diverge.  One loop iteration = two warp-wide phases:
//   node phase      every lane with pending inner nodes visits one 8-wide
//                   node: five 16-byte loads, eight child boxes decoded from
//                   8-bit planes with one FMA per plane;
//   triangle phase  the triangles of all lanes' hit leaves are pooled and
//                   spread over the 32 lanes (prefix sum + shuffle owner
//                   search), so a lane with 20 triangles does not idle the
//                   other 31.  Each result is folded into its owner's
//                   shared-memory key (ordered t << 32 | primitive) with a
//                   64-bit atomicMin, which is exactly the tie rule "lower t,
//                   then lower primitive"; the owner re-evaluates the winning
//                   triangle once for its barycentrics.
// The traversal stack holds (child base, hit mask, inner mask) groups: the
// top SSTACK entries live in shared memory, the rest in local memory;
// overflow is reported through the status word, never dropped.  In the
// batch's tail (ray pool exhausted), lanes without a ray help the busy
// lanes of their warp: each takes the bottom group of a busy lane's shared
// stack and walks it for that lane's ray (RTB_HELPERS).
//
// Box test robustness: t = q * (s/d) + (p - o)/d is evaluated with an
// absolute slack of 2^-22 |(p - o)/d| folded into the near/far offsets and
// a relative slack of 2^-21 on the far distance, which bounds every
// rounding of the decode, so a box that contains an accepted triangle hit
// is never culled.  Hit results are therefore defined by the triangle test
// alone: Moller-Trumbore in exact IEEE single precision (rt_common.cuh).
#include <algorithm>
#include <cfloat>

#include "rt_internal.h"
#include "rt_legacy.h"
#include "rt_trace.cuh"

// Analysis builds only (all default to 0; the release kernels are unchanged):
//   RTB_STATS     per-warp event counters (iterations, lanes per phase,
//                 triangle rounds) in g_trace_stats, read by rtStats_read;
//   RTB_DUP_NODE  every node visit done twice (the second result discarded
//                 through a value the compiler cannot know is zero), and
//   RTB_DUP_TRI   every triangle phase done twice (idempotent): the
//                 instruction count of one phase is then the difference to
//                 the release kernel's.
#ifndef RTB_STATS
#define RTB_STATS 0
#endif
#ifndef RTB_DUP_NODE
#define RTB_DUP_NODE 0
#endif
#ifndef RTB_DUP_TRI
#define RTB_DUP_TRI 0
#endif
// RTB_HELPERS: once the ray pool is exhausted, a lane left without a ray
// takes the oldest node group a busy lane of its warp keeps in shared
// memory and walks that subtree for the busy lane's ray (its triangles go
// to the ray's owner slot in the pooled phase, which keeps the closest hit
// exact: every triangle is still tested once and the minimum of the
// (t, primitive) keys does not depend on the order).  The owner writes the
// result once its own walk and all its helpers are done.  Not in the
// work-counting kernels, whose per-ray counts follow one walk order.
// 0: off; 1: closest hit only; 2: closest and any hit.  2 measured +1.8 %
// closest and +1.3 % any hit on 2M incoherent rays (warp iterations -4.8 %,
// lanes holding a ray at an iteration's start 28.6 -> 29.8 of 32) and
// steadier run to run.  Measured and left out: a victim with nothing
// stacked giving the far half of its current group (+1.1 / -0.6 %), and a
// warp vote that skips the owner-slot shuffle while no lane helps (+0.5 /
// -0.3 %: its register spills).
#ifndef RTB_HELPERS
#define RTB_HELPERS 2
#endif
// RTB_MID_REFILL: a lane whose ray has finished its traversal (no group,
// nothing stacked) takes the next ray at its next node visit instead of
// waiting for the iteration's end; the finished ray is parked in the lane's
// second shared-memory slot (its best key, barycentrics and output index)
// until the triangle phase has tested its pending triangles, then written.
// Pending triangle sets carry their ray's slot in the top bit of the
// record base.  Single-scene launches only, not the work-counting kernels.
#ifndef RTB_MID_REFILL
#define RTB_MID_REFILL 0
#endif
// launch modes with helpers (bit 1 << MODE_SINGLE / MODE_BATCH / MODE_WAVE):
// single scene only.  In the batch and wave modes the extra state spills
// (10-12 bytes) and the tail is a small part of their long launches: the
// 256-scene batched trace measured -4.5 % and the served waves -2 to -3 %.
#ifndef RTB_HELPERS_MODES
#define RTB_HELPERS_MODES 1
#endif

namespace rtb {

#if RTB_STATS
__device__ unsigned long long g_trace_stats[16];
#define RTB_STAT(k, v)                                                             \
    do {                                                                           \
        const unsigned long long _v = (unsigned long long)(v);                     \
        if (lane == 0 && _v) atomicAdd(&g_trace_stats[k], _v);                   \
    } while (0)
#else
#define RTB_STAT(k, v) \
    do {               \
    } while (0)
#endif

__device__ __forceinline__ void* ldg_ptr(const void* p) {
    return reinterpret_cast<void*>(__ldg(reinterpret_cast<const unsigned long long*>(p)));
}

// MODE_SINGLE: one scene, root 0, ray i -> rays[i], result i.
// MODE_BATCH: the structure holds several scenes (roots 0 .. nscenes-1); ray
//   i belongs to the scene s with ray_off[s] <= i < ray_off[s+1], starts at
//   root s, and reports primitives relative to tri_off[s].
// MODE_WAVE: a shared wavefront of `nscenes` segments (chunks of requests
//   against scenes resident in one arena); ray i belongs to the last segment
//   g with segs[g].first <= i, is read from segs[g].rays[i - first], starts
//   at node segs[g].root and is written to segs[g].out[i - first].
// T threads per CTA and SS shared stack entries per thread are template
// parameters so the batched form's autotuner can choose them; the CTA count
// the register budget must allow scales with T (the same 64 registers).
template <bool ANY, bool COUNT, int MODE, int NITERS, int T = TRACE_T, int SS = SSTACK>
__global__ void __launch_bounds__(T, (ANY ? TRACE_MINB_ANY : TRACE_MINB) * TRACE_T / T)
    k_trace_blas(const uint4* __restrict__ nodes, const float4* __restrict__ tris, const RtRay* __restrict__ rays,
                 int n, RtHit* __restrict__ hits, uint8_t* __restrict__ occ, uint32_t* __restrict__ counts,
                 int* __restrict__ work, int* __restrict__ status, const int* __restrict__ ray_off,
                 const int* __restrict__ tri_off, int nscenes, const WaveSeg* __restrict__ segs) {
    // ray slots per lane: the current ray, and with mid-iteration refill a
    // parked (finished) one; slot index = tag * T + thread
    constexpr bool MID = RTB_MID_REFILL && !COUNT && MODE == MODE_SINGLE;
    constexpr int NSL = MID ? 2 : 1;
    __shared__ uint2 sstack[SS][T];
    __shared__ unsigned long long s_key[NSL * T];  // a slot's best (ordered t, prim)
    __shared__ int s_rec[NSL * T];                 // set when a worker improved it (any hit: found)
    __shared__ float2 s_uv[NSL * T];               // barycentrics of the improved best
#if RTB_RAY_SMEM
    __shared__ float4 s_ray[NSL][2][T];            // each slot's ray, read by the lanes testing its triangles
#endif
    __shared__ int s_prev[MID ? T : 1];            // output index of the lane's parked ray, -1: none
    if (MID) s_prev[threadIdx.x] = -1;
    constexpr bool HELP =
        !COUNT && (ANY ? RTB_HELPERS >= 2 : RTB_HELPERS >= 1) && ((RTB_HELPERS_MODES >> MODE) & 1);
    constexpr bool PACK = (ANY ? RTB_PACK_ANY : RTB_PACK_CLOSEST) != 0;  // packed f32x2 plane distances
    static_assert(!HELP || RTB_RAY_SMEM, "helper lanes read the owner's ray from shared memory");
    static_assert(!MID || (RTB_RAY_SMEM && RTB_TWO_SETS), "parked rays are read from shared memory by set tag");
    // helpers per owner lane (low 16 bits) | HELP_OVF when a helper's stack overflowed
    constexpr int HELP_OVF = 1 << 16;
    __shared__ int s_help[HELP ? T : 1];
    if (HELP) s_help[threadIdx.x] = 0;
#if RTB_SLOTMASK
    __shared__ NodeLuts s_luts;
    init_node_luts(&s_luts);
    const NodeLuts* s_oct_perm = &s_luts;
#else
    const NodeLuts* s_oct_perm = nullptr;
#endif
    uint2 lstack[WalkT<T, SS>::L];
    const int lane = threadIdx.x & 31;
    const int wbase = threadIdx.x & ~31;
    // ray >= 0: this lane's own ray; -1: none; HELP: -2 - l when this lane
    // walks a subtree for the ray of lane l of its warp
    int ray = -1;
    bool exhausted = false;
    Ray r;
    WalkT<T, SS> w;
    float thit = 0.f, hu = 0.f, hv = 0.f;
    int hprim = -1;
    int prim_base = 0;
    int wseg = 0;
    uint32_t cn = 0, ct = 0;
    uint32_t tag = 0;  // slot of this lane's current ray (always 0 without MID)
    for (;;) {
        // ---- refill idle lanes ----
        const bool need = ray == -1 && !exhausted;
        const unsigned want = __ballot_sync(FULL_MASK, need);
        RTB_STAT(15, __popc(want));
        if (want) {
            const int leader = __ffs(want) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(work, __popc(want));
            base = __shfl_sync(FULL_MASK, base, leader);
            if (need) {
                const int ri = base + __popc(want & ((1u << lane) - 1));
                if (ri < n) {
                    uint32_t root = 0;
                    if (MODE == MODE_BATCH) {
                        int lo = 0, hi = nscenes - 1;  // last scene whose first ray <= ri
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (__ldg(ray_off + mid) <= ri) lo = mid;
                            else hi = mid - 1;
                        }
                        root = (uint32_t)lo;
                        prim_base = __ldg(tri_off + lo);
                    }
                    if (MODE == MODE_WAVE) {
                        int lo = 0, hi = nscenes - 1;  // last segment whose first ray <= ri
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if ((int)__ldg(&segs[mid].first) <= ri) lo = mid;
                            else hi = mid - 1;
                        }
                        wseg = lo;
                        root = __ldg(&segs[lo].root);
                        ray = ri - (int)__ldg(&segs[lo].first);
                        r = load_ray(reinterpret_cast<const RtRay*>(ldg_ptr(&segs[lo].rays)), ray);
                    } else {
                        ray = ri;
                        r = load_ray(rays, ri);
                    }
                    thit = r.tmax;
                    hprim = -1;
                    hu = hv = 0.f;
                    w.start();
#if RTB_RAY_SMEM
                    s_ray[tag][0][threadIdx.x] = make_float4(r.ox, r.oy, r.oz, r.tmin);
                    s_ray[tag][1][threadIdx.x] = make_float4(r.dx, r.dy, r.dz, r.tmax);
#endif
                    w.ng = make_uint2(root, (1u << r.oct) | (1u << 8));
                    cn = ct = 0;
                } else {
                    exhausted = true;
                }
            }
        }
        if (HELP) {
            // ---- tail: idle lanes take the oldest stacked group of a busy lane ----
            const bool idle = ray == -1 && exhausted;
            const unsigned idles = __ballot_sync(FULL_MASK, idle);
            const bool can = idles && ray != -1 && w.sp > w.sb && w.sb < WalkT<T, SS>::S;
            const unsigned vict = idles ? __ballot_sync(FULL_MASK, can) : 0u;
            if (vict) {
                const int nst = min(__popc(idles), __popc(vict));
                const int irank = __popc(idles & ((1u << lane) - 1));
                const bool thief = idle && irank < nst;
                const bool given = can && __popc(vict & ((1u << lane) - 1)) < nst;
                const int v = thief ? (int)nth_set_bit(vict, (uint32_t)irank) : lane;
                // the victim's part: its bottom stacked group (from its own shared column)
                uint2 give = make_uint2(0u, 0u);
                if (given) {
                    give = sstack[w.sb][threadIdx.x];
                    w.sb++;
                }
                const uint32_t gx = __shfl_sync(FULL_MASK, give.x, v), gy = __shfl_sync(FULL_MASK, give.y, v);
                const int vslot = __shfl_sync(FULL_MASK, ray >= 0 ? lane : -2 - ray, v);
                const float vthit = __shfl_sync(FULL_MASK, thit, v);
                const uint32_t vtag = MID ? __shfl_sync(FULL_MASK, tag, v) : 0u;
                if (thief) {
                    ray = -2 - vslot;
                    if (MID) tag = vtag;  // the owner's slot
                    r = make_ray(s_ray[vtag][0][wbase + vslot], s_ray[vtag][1][wbase + vslot]);
                    thit = vthit;
                    hprim = -1;
                    w.start();
                    w.ng = make_uint2(gx, gy);
                    atomicAdd(&s_help[wbase + vslot], 1);
                }
            }
        }
        if (__all_sync(FULL_MASK, ray == -1)) break;
        RTB_STAT(0, 1);
        RTB_STAT(1, __popc(__ballot_sync(FULL_MASK, ray >= 0)));
        // ---- node phase ----
        uint32_t tri_base = 0, tmask = 0;
#if RTB_TWO_SETS
        uint32_t tri_base2 = 0, tmask2 = 0;  // a second visit's leaves while the first set waits
#else
        constexpr uint32_t tmask2 = 0;
#endif
#if RTB_THREE_SETS
        uint32_t tri_base3 = 0, tmask3 = 0;  // and a third (RTB_THREE_SETS)
#define RTB_LAST_SET tmask3
#else
        constexpr uint32_t tmask3 = 0;
#define RTB_LAST_SET tmask2
#endif
        bool overflow = false;
#pragma unroll 1
        for (int it = 0; it < NITERS; it++) {
#if RTB_STATS
            {
#if RTB_TWO_SETS
                const bool visit = ray >= 0 && RTB_LAST_SET == 0 && !overflow && (w.ng.y & 0xFFu);
#else
                const bool visit = ray >= 0 && tmask == 0 && !overflow && (w.ng.y & 0xFFu);
#endif
                const unsigned act = __ballot_sync(FULL_MASK, visit);
                RTB_STAT(2 + 2 * it, act ? 1 : 0);  // visit it: warp executions (it < 5)
                RTB_STAT(3 + 2 * it, __popc(act));  //           lanes
            }
#endif
            if (MID && it > 0) {
                // lanes whose own ray has finished its traversal take the next ray
                const bool fin = ray >= 0 && !exhausted && !overflow && RTB_LAST_SET == 0 &&
                                 (w.ng.y & 0xFFu) == 0 && w.sp == w.sb && s_prev[threadIdx.x] < 0;
                const unsigned fwant = __ballot_sync(FULL_MASK, fin);
                if (fwant) {
                    const int leader = __ffs(fwant) - 1;
                    int base = 0;
                    if (lane == leader) base = atomicAdd(work, __popc(fwant));
                    base = __shfl_sync(FULL_MASK, base, leader);
                    if (fin) {
                        const int ri = base + __popc(fwant & ((1u << lane) - 1));
                        if (ri < n) {
                            // park the finished ray: its best so far stays in its slot
                            const int ps = (int)tag * T + threadIdx.x;
                            if (ANY) {
                                s_rec[ps] = 0;
                            } else {
                                s_key[ps] = ((unsigned long long)f2ord(thit) << 32) |
                                            (uint32_t)(hprim >= 0 ? hprim : -1);
                                s_uv[ps] = make_float2(hu, hv);
                            }
                            s_prev[threadIdx.x] = ray;
                            tag ^= 1u;
                            ray = ri;
                            r = load_ray(rays, ri);
                            thit = r.tmax;
                            hprim = -1;
                            hu = hv = 0.f;
                            w.start();
                            s_ray[tag][0][threadIdx.x] = make_float4(r.ox, r.oy, r.oz, r.tmin);
                            s_ray[tag][1][threadIdx.x] = make_float4(r.dx, r.dy, r.dz, r.tmax);
                            w.ng = make_uint2(0u, (1u << r.oct) | (1u << 8));
                        } else {
                            exhausted = true;
                        }
                    }
                }
            }
#if RTB_TWO_SETS
#if RTB_VISIT_VOTE
            // later visits only while some lane can still take one
            if (it > 0 && !__any_sync(FULL_MASK, ray >= 0 && RTB_LAST_SET == 0 && !overflow && (w.ng.y & 0xFFu)))
                break;
#endif
            if (ray != -1 && RTB_LAST_SET == 0 && !overflow && (w.ng.y & 0xFFu)) {
#else
            if (ray != -1 && tmask == 0 && !overflow && (w.ng.y & 0xFFu)) {
#endif
                uint32_t hitsm = w.ng.y & 0xFFu;
                const uint32_t imask = (w.ng.y >> 8) & 0xFFu;
                const int k = __ffs(hitsm) - 1;
                hitsm &= hitsm - 1;
                const uint32_t slot = (uint32_t)k ^ r.oct;
                const uint32_t ni = w.ng.x + __popc(imask & ((1u << slot) - 1));
                if (hitsm && !w.push(make_uint2(w.ng.x, hitsm | (imask << 8)), sstack, lstack)) overflow = true;
                if (COUNT) cn++;
                uint32_t nmask;
#if RTB_TWO_SETS
                uint32_t vb, vm;
                visit_node<RTB_SLOTMASK, PACK>(nodes + (size_t)ni * 5, r, thit, nmask, vb, vm, w.ng, s_oct_perm);
                if (MID) vb |= tag << 31;  // the set's ray slot
                if (tmask == 0) {
                    tri_base = vb;
                    tmask = vm;
#if RTB_THREE_SETS
                } else if (tmask2 == 0) {
                    tri_base2 = vb;
                    tmask2 = vm;
                } else {
                    tri_base3 = vb;
                    tmask3 = vm;
                }
#else
                } else {
                    tri_base2 = vb;
                    tmask2 = vm;
                }
#endif
#else
                visit_node<RTB_SLOTMASK, PACK>(nodes + (size_t)ni * 5, r, thit, nmask, tri_base, tmask, w.ng, s_oct_perm);
#endif
#if RTB_DUP_NODE
                {
                    uint32_t nm2, tb2, tm2;
                    uint2 ng2;
                    visit_node<RTB_SLOTMASK, PACK>(nodes + (size_t)ni * 5, r, thit, nm2, tb2, tm2, ng2, s_oct_perm);
                    const uint32_t z = (uint32_t)(n >> 31);  // 0 for n >= 0, unknown at compile time
                    tmask |= tm2 & z;
                    tri_base |= tb2 & z;
                    w.ng.x |= ng2.x & z;
                    w.ng.y |= ng2.y & z;
                }
#endif
                prefetch_next(nodes, w.ng, r.oct);
#if RTB_TWO_SETS
                if (NITERS > 1 && (w.ng.y & 0xFFu) == 0 && w.sp > w.sb) {
#else
                if (NITERS > 1 && tmask == 0 && (w.ng.y & 0xFFu) == 0 && w.sp > w.sb) {
#endif
                    w.ng = w.pop(sstack, lstack);
                }
            }
        }
        // ---- triangle phase: pooled over the warp ----
        const int cnt = __popc(tmask) + __popc(tmask2) + __popc(tmask3);
        int incl = cnt, total = 0;
        // RTB_TRI_VOTE: one warp vote skips the scan when no lane holds triangles
        if (!RTB_TRI_VOTE || __any_sync(FULL_MASK, tmask != 0)) {
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULL_MASK, incl, o);
                if (lane >= o) incl += y;
            }
            total = __shfl_sync(FULL_MASK, incl, 31);
        }
        bool found_any = false;
        RTB_STAT(12, total ? 1 : 0);
        RTB_STAT(13, (total + 31) / 32);
        RTB_STAT(14, total);
#if RTB_DUP_TRI
#pragma unroll 1
        for (int rep = 0; rep < 2; rep++)
#endif
        if (total) {
            const int excl = incl - cnt;
            if (COUNT) ct += cnt;
            const int cur_slot = (int)tag * T + threadIdx.x;
            if (!ANY) {
                s_key[cur_slot] = ((unsigned long long)f2ord(thit) << 32) | (uint32_t)(hprim >= 0 ? hprim : -1);
                s_rec[cur_slot] = -1;
            } else {
                s_rec[cur_slot] = 0;
            }
            __syncwarp();
            const int kslot = HELP && ray < -1 ? -2 - ray : lane;  // whose ray this lane's triangles belong to
            for (int base = 0; base < total; base += 32) {
                const int g = base + lane;
                // owner = first lane whose inclusive count exceeds g
                int o = 0;
#pragma unroll
                for (int s = 16; s; s >>= 1) {
                    const int v = __shfl_sync(FULL_MASK, incl, o + s - 1);
                    if (v <= g) o += s;
                }
                o = min(o, 31);
                const int k0 = g - __shfl_sync(FULL_MASK, excl, o);
                const int ko = HELP ? __shfl_sync(FULL_MASK, kslot, o) : o;  // the triangle's ray slot
#if RTB_TWO_SETS
                uint32_t om = __shfl_sync(FULL_MASK, tmask, o);
                uint32_t ob = __shfl_sync(FULL_MASK, tri_base, o);
                const uint32_t om2 = __shfl_sync(FULL_MASK, tmask2, o);
                const uint32_t ob2 = __shfl_sync(FULL_MASK, tri_base2, o);
                const int c1 = __popc(om);
#if RTB_THREE_SETS
                const uint32_t om3 = __shfl_sync(FULL_MASK, tmask3, o);
                const uint32_t ob3 = __shfl_sync(FULL_MASK, tri_base3, o);
                const int c12 = c1 + __popc(om2);
                const int k = k0 < c1 ? k0 : (k0 < c12 ? k0 - c1 : k0 - c12);
                if (k0 >= c12) {
                    om = om3;
                    ob = ob3;
                } else if (k0 >= c1) {
                    om = om2;
                    ob = ob2;
                }
#else
                const int k = k0 < c1 ? k0 : k0 - c1;
                if (k0 >= c1) {
                    om = om2;
                    ob = ob2;
                }
#endif
#else
                const int k = k0;
                const uint32_t om = __shfl_sync(FULL_MASK, tmask, o);
                uint32_t ob = __shfl_sync(FULL_MASK, tri_base, o);
#endif
                // the set's ray slot (MID: top bit of the record base)
                const uint32_t otag = MID ? ob >> 31 : 0u;
                if (MID) ob &= 0x7FFFFFFFu;
                const int kidx = (int)otag * T + wbase + ko;
#if RTB_RAY_SMEM
                const float4 ro = s_ray[otag][0][wbase + ko], rd = s_ray[otag][1][wbase + ko];
                const float ox = ro.x, oy = ro.y, oz = ro.z, tmn = ro.w;
                const float dx = rd.x, dy = rd.y, dz = rd.z, tmx = rd.w;
#else
                const float ox = __shfl_sync(FULL_MASK, r.ox, o), oy = __shfl_sync(FULL_MASK, r.oy, o),
                            oz = __shfl_sync(FULL_MASK, r.oz, o);
                const float dx = __shfl_sync(FULL_MASK, r.dx, o), dy = __shfl_sync(FULL_MASK, r.dy, o),
                            dz = __shfl_sync(FULL_MASK, r.dz, o);
                const float tmn = __shfl_sync(FULL_MASK, r.tmin, o), tmx = __shfl_sync(FULL_MASK, r.tmax, o);
#endif
                unsigned long long key = ~0ull;
                float u = 0.f, v = 0.f;
                if (g < total) {
                    const int rec = (int)ob + (int)nth_set_bit(om, (uint32_t)k);
                    const float4* tp = tris + (size_t)rec * 3;
                    const float4 A = ld_tri(tp), B = ld_tri(tp + 1), Cc = ld_tri(tp + 2);
                    float t;
                    if (intersect_tri(ox, oy, oz, dx, dy, dz, A, B, Cc, t, u, v) && t > tmn && t < tmx) {
                        if (ANY) s_rec[kidx] = 1;
                        else key = ((unsigned long long)f2ord(t) << 32) | (uint32_t)__float_as_int(A.w);
                    }
                }
                if (!ANY) {
                    if (key != ~0ull) atomicMin(&s_key[kidx], key);
                    __syncwarp();
                    // the unique winner (keys are distinct per ray) publishes its barycentrics
                    if (key != ~0ull && s_key[kidx] == key) {
                        s_rec[kidx] = 1;
                        s_uv[kidx] = make_float2(u, v);
                    }
                    __syncwarp();
                }
            }
            __syncwarp();
            const int tb = (int)tag * T;
            if (ANY) {
                found_any = s_rec[tb + (HELP && ray < -1 ? wbase - 2 - ray : (int)threadIdx.x)] != 0;
            } else if (HELP && ray < -1) {
                thit = ord2f((uint32_t)(s_key[tb + wbase - 2 - ray] >> 32));  // the owner's best so far culls
            } else if (s_rec[tb + threadIdx.x] >= 0) {
                // a new closest hit for this lane
                const unsigned long long key = s_key[tb + threadIdx.x];
                const float2 uv = s_uv[tb + threadIdx.x];
                thit = ord2f((uint32_t)(key >> 32));
                hprim = (int)(uint32_t)key;
                hu = uv.x;
                hv = uv.y;
            }
        }
        if (MID) {
            // the parked ray's triangles are tested: its slot holds the result
            const int pr = s_prev[threadIdx.x];
            if (pr >= 0) {
                const int ps = (int)(tag ^ 1u) * T + threadIdx.x;
                if (ANY) {
                    occ[pr] = s_rec[ps] != 0 ? 1 : 0;
                } else {
                    const unsigned long long key = s_key[ps];
                    const float2 uv = s_uv[ps];
                    const int pp = (int)(uint32_t)key;
                    const float4 hv4 = make_float4(pp >= 0 ? ord2f((uint32_t)(key >> 32)) : __int_as_float(0x7f800000),
                                                   __int_as_float(pp >= 0 ? pp : -1), pp >= 0 ? uv.x : 0.f,
                                                   pp >= 0 ? uv.y : 0.f);
#if RTB_RAY_CS
                    __stcs(reinterpret_cast<float4*>(hits) + pr, hv4);
#else
                    reinterpret_cast<float4*>(hits)[pr] = hv4;
#endif
                }
                s_prev[threadIdx.x] = -1;
            }
        }
        // ---- advance / finish ----
        bool owner_done = false;
        if (ray != -1) {
            bool done = overflow || (ANY && found_any);
            if (!done && (w.ng.y & 0xFFu) == 0) {
                if (w.sp == w.sb) {
                    done = true;
                } else {
                    w.ng = w.pop(sstack, lstack);
                    prefetch_next(nodes, w.ng, r.oct);
                }
            }
            if (HELP && ray < -1) {
                if (done) {  // subtree walked (or the ray already occluded): leave the owner
                    if (overflow) atomicOr(&s_help[wbase - 2 - ray], HELP_OVF);
                    atomicSub(&s_help[wbase - 2 - ray], 1);
                    ray = -1;
                }
            } else {
                owner_done = done;
            }
        }
        if (HELP) {
            __syncwarp();  // helpers' departures are visible to their owners
            if (owner_done) {
                const int hs = s_help[threadIdx.x];
                if (hs & (HELP_OVF - 1)) {
                    // own walk over, helpers still out: keep what decided it and wait
                    if (overflow) atomicOr(&s_help[threadIdx.x], HELP_OVF);
                    if (ANY && found_any) hprim = 0;  // any hit: found (hprim is otherwise unused)
                    w.ng.y &= ~0xFFu;
                    w.sp = w.sb;
                    owner_done = false;
                } else {
                    overflow = overflow || (hs & HELP_OVF);
                    if (ANY) found_any = found_any || hprim >= 0;
                    s_help[threadIdx.x] = 0;
                }
            }
        } else {
            owner_done = ray >= 0 && owner_done;
        }
        if (owner_done) {
            {
                if (overflow) {
                    atomicOr(status, RT_STATUS_STACK);
                    hprim = -1;
                    found_any = false;
                }
                if (MODE == MODE_WAVE) {
                    if (ANY) occ = reinterpret_cast<uint8_t*>(ldg_ptr(&segs[wseg].out));
                    else hits = reinterpret_cast<RtHit*>(ldg_ptr(&segs[wseg].out));
                }
                if (ANY) {
                    occ[ray] = found_any ? 1 : 0;
                } else {
                    const float4 hv4 = make_float4(hprim >= 0 ? thit : __int_as_float(0x7f800000),
                                                   __int_as_float(hprim >= 0 ? hprim - prim_base : -1),
                                                   hprim >= 0 ? hu : 0.f, hprim >= 0 ? hv : 0.f);
#if RTB_RAY_CS
                    __stcs(reinterpret_cast<float4*>(hits) + ray, hv4);
#else
                    reinterpret_cast<float4*>(hits)[ray] = hv4;
#endif
                }
                if (COUNT) reinterpret_cast<uint2*>(counts)[ray] = make_uint2(cn, ct);
                ray = -1;
            }
        }
    }
}

template <class K>
static int persistent_grid(K kernel, int threads) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    return per_sm * num_sms();
}

#if RTB_STATS
extern "C" int rtStats_read(unsigned long long* out16, int reset) {
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpyFromSymbol(out16, g_trace_stats, sizeof(unsigned long long) * 16) != cudaSuccess)
        return -1;
    if (reset) {
        static const unsigned long long zero[16] = {};
        if (cudaMemcpyToSymbol(g_trace_stats, zero, sizeof(zero)) != cudaSuccess) return -1;
    }
    return 0;
}
#endif

int launch_trace_blas(const Bvh8Device& b, const RtRay* rays, int n, RtHit* hits, uint8_t* occ,
                      uint32_t* counts, int* work, int* status, cudaStream_t s) {
    const uint4* nodes = reinterpret_cast<const uint4*>(b.nodes.p);
    const float4* tris = reinterpret_cast<const float4*>(b.tris.p);
    constexpr int NI = RTB_NODE_ITERS;
    if (counts) {
        if (occ) {
            static const int g = persistent_grid(k_trace_blas<true, true, MODE_SINGLE, NI>, TRACE_T);
            k_trace_blas<true, true, MODE_SINGLE, NI><<<g, TRACE_T, 0, s>>>(nodes, tris, rays, n, hits, occ, counts, work,
                                                                     status, nullptr, nullptr, 1, nullptr);
        } else {
            static const int g = persistent_grid(k_trace_blas<false, true, MODE_SINGLE, NI>, TRACE_T);
            k_trace_blas<false, true, MODE_SINGLE, NI><<<g, TRACE_T, 0, s>>>(nodes, tris, rays, n, hits, occ, counts, work,
                                                                      status, nullptr, nullptr, 1, nullptr);
        }
    } else if (occ) {
        static const int g = persistent_grid(k_trace_blas<true, false, MODE_SINGLE, NI>, TRACE_T);
        k_trace_blas<true, false, MODE_SINGLE, NI><<<g, TRACE_T, 0, s>>>(nodes, tris, rays, n, hits, occ, counts, work,
                                                                  status, nullptr, nullptr, 1, nullptr);
    } else {
        static const int g = persistent_grid(k_trace_blas<false, false, MODE_SINGLE, NI>, TRACE_T);
        k_trace_blas<false, false, MODE_SINGLE, NI><<<g, TRACE_T, 0, s>>>(nodes, tris, rays, n, hits, occ, counts, work,
                                                                   status, nullptr, nullptr, 1, nullptr);
    }
    return RT_CUDA(cudaGetLastError()) ? RT_OK : RT_ERR_CUDA;
}

// Many scenes in one persistent launch, in the shape the batched form's
// autotuner chose: persistent worker warps per SM, node visits per
// iteration, threads per CTA and shared stack entries per thread.  The
// instantiated shapes are the tuner's candidates: (block, shared stack) in
// {(128, 8), (64, 8), (256, 8), (128, 4), (128, 12)}, node visits 2 or 4
// (3 also at (128, 8)); other values fall back to the nearest (128, 8) one.
template <bool ANY, int NI, int T, int SS>
static void launch_batch(int warps_per_sm, const uint4* nodes, const float4* tris, const RtRay* rays, int n,
                         RtHit* hits, uint8_t* occ, int* work, int* status, const int* ray_off, const int* tri_off,
                         int nscenes, cudaStream_t s) {
    const int max_ctas = (ANY ? TRACE_MINB_ANY : TRACE_MINB) * TRACE_T / T;
    const int ctas = std::max(1, std::min(warps_per_sm * 32 / T, max_ctas));
    k_trace_blas<ANY, false, MODE_BATCH, NI, T, SS><<<ctas * num_sms(), T, 0, s>>>(
        nodes, tris, rays, n, hits, occ, nullptr, work, status, ray_off, tri_off, nscenes, nullptr);
}

template <bool ANY, int NI>
static void launch_batch_shape(const BatchShape& sh, const uint4* nodes, const float4* tris, const RtRay* rays, int n,
                               RtHit* hits, uint8_t* occ, int* work, int* status, const int* ray_off,
                               const int* tri_off, int nscenes, cudaStream_t s) {
#define RTB_BATCH_ARGS sh.warps_per_sm, nodes, tris, rays, n, hits, occ, work, status, ray_off, tri_off, nscenes, s
    if (sh.block == 64 && sh.shared_stack == 8) launch_batch<ANY, NI, 64, 8>(RTB_BATCH_ARGS);
    else if (sh.block == 256 && sh.shared_stack == 8) launch_batch<ANY, NI, 256, 8>(RTB_BATCH_ARGS);
    else if (sh.block == 128 && sh.shared_stack == 4) launch_batch<ANY, NI, 128, 4>(RTB_BATCH_ARGS);
    else if (sh.block == 128 && sh.shared_stack == 12) launch_batch<ANY, NI, 128, 12>(RTB_BATCH_ARGS);
    else launch_batch<ANY, NI, 128, 8>(RTB_BATCH_ARGS);
#undef RTB_BATCH_ARGS
}

int launch_trace_multi(const Bvh8Device& b, const RtRay* rays, int n, const int* ray_off, const int* tri_off,
                       int nscenes, RtHit* hits, uint8_t* occ, int* work, int* status, const BatchShape& sh,
                       cudaStream_t s) {
    const uint4* nodes = reinterpret_cast<const uint4*>(b.nodes.p);
    const float4* tris = reinterpret_cast<const float4*>(b.tris.p);
    const bool base_shape = sh.block == 128 && sh.shared_stack == 8;
    if (occ) {
        if (sh.node_iters == 3 && base_shape)
            launch_batch<true, 3, 128, 8>(sh.warps_per_sm, nodes, tris, rays, n, hits, occ, work, status, ray_off,
                                          tri_off, nscenes, s);
        else if (sh.node_iters <= 2)
            launch_batch_shape<true, 2>(sh, nodes, tris, rays, n, hits, occ, work, status, ray_off, tri_off, nscenes, s);
        else
            launch_batch_shape<true, 4>(sh, nodes, tris, rays, n, hits, occ, work, status, ray_off, tri_off, nscenes, s);
    } else {
        if (sh.node_iters == 3 && base_shape)
            launch_batch<false, 3, 128, 8>(sh.warps_per_sm, nodes, tris, rays, n, hits, occ, work, status, ray_off,
                                           tri_off, nscenes, s);
        else if (sh.node_iters <= 2)
            launch_batch_shape<false, 2>(sh, nodes, tris, rays, n, hits, occ, work, status, ray_off, tri_off, nscenes,
                                         s);
        else
            launch_batch_shape<false, 4>(sh, nodes, tris, rays, n, hits, occ, work, status, ray_off, tri_off, nscenes,
                                         s);
    }
    return RT_CUDA(cudaGetLastError()) ? RT_OK : RT_ERR_CUDA;
}

// One shared wavefront: `n` rays over `nseg` segments, all of one kind.
int launch_trace_wave(const uint4* nodes, const float4* tris, const WaveSeg* segs, int nseg, int n, bool any,
                      int* work, int* status, int ctas_per_sm, cudaStream_t s) {
    const int g = std::max(1, std::min(ctas_per_sm, any ? TRACE_MINB_ANY : TRACE_MINB)) * num_sms();
    if (any)
        k_trace_blas<true, false, MODE_WAVE, RTB_NODE_ITERS><<<g, TRACE_T, 0, s>>>(nodes, tris, nullptr, n, nullptr, nullptr,
                                                                     nullptr, work, status, nullptr, nullptr, nseg,
                                                                     segs);
    else
        k_trace_blas<false, false, MODE_WAVE, RTB_NODE_ITERS><<<g, TRACE_T, 0, s>>>(nodes, tris, nullptr, n, nullptr, nullptr,
                                                                      nullptr, work, status, nullptr, nullptr, nseg,
                                                                      segs);
    return RT_CUDA(cudaGetLastError()) ? RT_OK : RT_ERR_CUDA;
}

// Copies one scene's 8-wide nodes into an arena at node offset `node_off`,
// rebasing child and triangle bases by node_off and tri_off.
__global__ void k_rebase_nodes(const uint4* __restrict__ src, uint4* __restrict__ dst, int count, uint32_t node_off,
                               uint32_t tri_off) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint4* a = src + (size_t)i * 5;
    uint4* b = dst + (size_t)i * 5;
    uint4 w1 = a[1];
    w1.x += node_off;
    w1.y += tri_off;
    b[0] = a[0];
    b[1] = w1;
    b[2] = a[2];
    b[3] = a[3];
    b[4] = a[4];
}

void launch_rebase_nodes(const void* src, void* dst, int count, uint32_t node_off, uint32_t tri_off,
                         cudaStream_t s) {
    if (count <= 0) return;
    k_rebase_nodes<<<(count + 255) / 256, 256, 0, s>>>(reinterpret_cast<const uint4*>(src),
                                                         reinterpret_cast<uint4*>(dst), count, node_off, tri_off);
}

}  // namespace rtb
