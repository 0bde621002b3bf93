// rt_trace.cuh -- traversal building blocks shared by the single-level,
// two-level and wavefront kernels.
#pragma once
#include "rt_common.cuh"

namespace rtb {

constexpr unsigned FULL_MASK = 0xFFFFFFFFu;
// Build-time knobs of the traversal kernels; the defaults are the measured
// best on B200 for 2M incoherent rays (64 registers -> 32 warps per SM; two
// pending triangle sets and four node visits per lane between pooled
// triangle phases; 3-input min/max; the owner's ray read from shared memory
// in the triangle phase, +1.4 %).
// Measured and rejected: L1 prefetch of the next node (-10%), branchless
// child masks (-2%), folding the bias of an older 2^23 + byte decode into
// the offsets (0%),
// ray reordering by origin Morton code / direction octant (+1%, scene is
// L2-resident), leaf sizes 2 and 3 (-3%, -1%).
#ifndef RTB_TRACE_MINB
#define RTB_TRACE_MINB 8
#endif
// any-hit CTAs per SM: with two pending triangle sets and four node
// visits, 8 (64 registers, no spills) measured +4.6 % over 9 (56 registers,
// a few bytes spilled); 9 had been +1.9 % over 8 with one set and 2 visits
#ifndef RTB_TRACE_MINB_ANY
#define RTB_TRACE_MINB_ANY 8
#endif
#ifndef RTB_SSTACK
#define RTB_SSTACK 8
#endif
#ifndef RTB_PREFETCH
#define RTB_PREFETCH 0
#endif
#ifndef RTB_BRANCHLESS
#define RTB_BRANCHLESS 0
#endif
// node visits per lane between pooled triangle phases (with two pending
// triangle sets, RTB_TWO_SETS): 4 measured best on 2M incoherent rays
// (closest hit +9.5 %, any hit +6.7 % over 2 visits and one set; 3: +8.9 /
// +4.1 %; 6: +3.5 / +0.7 %)
#ifndef RTB_NODE_ITERS
#define RTB_NODE_ITERS 4
#endif
#ifndef RTB_MAX3
#define RTB_MAX3 1
#endif
// L1 eviction priority of the traversal's loads (0: plain non-coherent
// loads).  Rays and hits are touched once and are streamed (measured
// neutral: +0.1 % closest hit on average over seven alternating pairs, each
// pair within +-1 %).  Measured and left off: triangle records not
// allocated in L1 (-2 %), nodes kept last (mixed, -0.4 % to +0.5 %).
#ifndef RTB_TRI_NA
#define RTB_TRI_NA 0
#endif
#ifndef RTB_NODE_EL
#define RTB_NODE_EL 0
#endif
#ifndef RTB_RAY_CS
#define RTB_RAY_CS 1
#endif
#ifndef RTB_TRI_VOTE
#define RTB_TRI_VOTE 0
#endif
// pooled triangle phase reads the owner's ray from shared memory (1) or
// gathers it with eight shuffles (0)
#ifndef RTB_RAY_SMEM
#define RTB_RAY_SMEM 1
#endif

// min/max of three floats, NaN operands ignored like fminf/fmaxf
// (sm_100 has three-input FMNMX).
__device__ __forceinline__ float max3f(float a, float b, float c) {
#if RTB_MAX3
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
#else
    return fmaxf(fmaxf(a, b), c);
#endif
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
#if RTB_MAX3
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
#else
    return fminf(fminf(a, b), c);
#endif
}
constexpr int TRACE_T = 128;               // threads per persistent CTA
constexpr int TRACE_MINB = RTB_TRACE_MINB; // CTAs per SM the register budget must allow
constexpr int TRACE_MINB_ANY = RTB_TRACE_MINB_ANY;
constexpr int SSTACK = RTB_SSTACK;         // stack entries per thread in shared memory
// Stack entries per ray in total (shared + local).  64 holds any tree the
// builder makes (validation rejects deeper ones); a test build lowers it to
// reach the overflow path, which reports RT_ERR_STACK.
#ifndef RTB_STACK_TOTAL
#define RTB_STACK_TOTAL 64
#endif
static_assert(RTB_STACK_TOTAL > RTB_SSTACK, "the local part of the stack needs at least one entry");
constexpr int LSTACK = RTB_STACK_TOTAL - SSTACK;  // further entries in local memory
constexpr int SSTACK_TOTAL = SSTACK + LSTACK;
constexpr int RT_STATUS_STACK = 1;
constexpr int RT_STATUS_TIMEOUT = 2;

struct Ray {
    float ox, oy, oz, tmin;
    float dx, dy, dz, tmax;
    float ix, iy, iz;  // box-test reciprocal direction (see guard_rcp)
    uint32_t oct;      // sign bits of ix, iy, iz: x -> 1, y -> 2, z -> 4
};

// Reciprocal direction for the box test only.  A component with |d| <= 2^-64
// (an exact zero included) is replaced by +-2^-64 keeping its sign, so the
// slab arithmetic stays finite (1/0 = inf would turn q*S + O into NaN and
// silently disable culling on that axis).  The box offsets carry an absolute
// slack of 2^-22 |(p - o)/d|, which for such an axis is |p - o| * 2^42 and
// covers the drift of the guarded direction over any finite scene, so the
// test stays conservative.  The triangle test uses the true direction.
__device__ __forceinline__ float guard_rcp(float d) {
    return __frcp_rn(fabsf(d) > 0x1p-64f ? d : copysignf(0x1p-64f, d));
}

__device__ __forceinline__ Ray make_ray(float4 a, float4 b) {
    Ray r;
    r.ox = a.x; r.oy = a.y; r.oz = a.z; r.tmin = a.w;
    r.dx = b.x; r.dy = b.y; r.dz = b.z; r.tmax = b.w;
    r.ix = guard_rcp(r.dx);
    r.iy = guard_rcp(r.dy);
    r.iz = guard_rcp(r.dz);
    r.oct = (signbit(r.ix) ? 1u : 0u) | (signbit(r.iy) ? 2u : 0u) | (signbit(r.iz) ? 4u : 0u);
    return r;
}

__device__ __forceinline__ Ray load_ray(const RtRay* rays, int i) {
    const float4* p = reinterpret_cast<const float4*>(rays + i);
#if RTB_RAY_CS
    return make_ray(__ldcs(p), __ldcs(p + 1));
#else
    return make_ray(__ldg(p), __ldg(p + 1));
#endif
}

// One 16-byte word of a triangle record / of a node (see RTB_TRI_NA, RTB_NODE_EL).
__device__ __forceinline__ float4 ld_tri(const float4* p) {
#if RTB_TRI_NA
    float4 v;
    asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p));
    return v;
#else
    return __ldg(p);
#endif
}
__device__ __forceinline__ uint4 ld_node(const uint4* p) {
#if RTB_NODE_EL
    uint4 v;
    asm("ld.global.nc.L1::evict_last.v4.u32 {%0, %1, %2, %3}, [%4];"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p));
    return v;
#else
    return __ldg(p);
#endif
}

// Position of the k-th (0-based) set bit of m (k < popc(m)).  A hit leaf's
// triangles are one contiguous run of bits, so the common case is
// ffs - 1 + k; otherwise a five-step popcount search.  Measured +3 % over
// __fns on the incoherent workload.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, uint32_t k) {
    const uint32_t lo = __ffs(m) - 1, run = m >> lo;
    if ((run & (run + 1)) == 0) return lo + k;
    uint32_t pos = 0, c;
    c = __popc(m & 0xFFFFu);
    if (k >= c) { k -= c; pos += 16; m >>= 16; }
    c = __popc(m & 0xFFu);
    if (k >= c) { k -= c; pos += 8; m >>= 8; }
    c = __popc(m & 0xFu);
    if (k >= c) { k -= c; pos += 4; m >>= 4; }
    c = __popc(m & 0x3u);
    if (k >= c) { k -= c; pos += 2; m >>= 2; }
    if (k >= (m & 1u)) pos += 1;
    return pos;
}

// RTB_SLOTMASK: the node test keeps one hit bit per child slot (a
// predicated OR, no branch), takes a leaf's triangle bits with one
// predicated OR, and moves the inner hits into the ray's octant order once
// per node with a table lookup (oct_perm, 2 KB of shared memory per CTA)
// instead of a shift per child.  1: a leaf's bits from bmsk of its meta
// byte; 2: from a 256-entry table indexed by the meta byte (1 KB of shared
// memory; inner slots' meta 0xFF and empty slots' 0 map to no bits).
#ifndef RTB_SLOTMASK
#define RTB_SLOTMASK 0
#endif
// RTB_TWO_SETS: a lane keeps up to two pending triangle sets, so a node
// visit that finds leaves does not stop the lane's next visit (measured
// +3 % closest and any hit at 2 visits, and what makes more visits pay).
#ifndef RTB_TWO_SETS
#define RTB_TWO_SETS 1
#endif
// RTB_THREE_SETS (with RTB_TWO_SETS): a third pending set.
#ifndef RTB_THREE_SETS
#define RTB_THREE_SETS 0
#endif
// RTB_VISIT_VOTE (with RTB_TWO_SETS): the node visits after the first stop
// as soon as no lane of the warp can take one (both sets pending or no node
// left), so RTB_NODE_ITERS can be a generous cap.
#ifndef RTB_VISIT_VOTE
#define RTB_VISIT_VOTE 0
#endif
constexpr int OCT_PERM_BYTES = 8 * 256;
// Lookup tables of the node test in shared memory (RTB_SLOTMASK).
struct NodeLuts {
    uint32_t meta_run[256];        // meta byte -> triangle bits of the leaf slot
    uint8_t oct_perm[OCT_PERM_BYTES];  // (o << 8) | x -> x with bit i moved to bit i ^ o
};
// Fills the tables; called by every thread of the CTA before its first node visit.
__device__ __forceinline__ void init_node_luts(NodeLuts* t) {
    for (int idx = threadIdx.x; idx < OCT_PERM_BYTES; idx += blockDim.x) {
        const uint32_t o = (uint32_t)idx >> 8, x = (uint32_t)idx & 0xFFu;
        uint32_t y = 0;
        for (uint32_t i = 0; i < 8; i++) y |= ((x >> i) & 1u) << (i ^ o);
        t->oct_perm[idx] = (uint8_t)y;
    }
    for (int m = threadIdx.x; m < 256; m += blockDim.x) {
        // leaf: count << 5 | offset; 0xFF marks an inner child, 0 an empty slot
        const uint32_t off = (uint32_t)m & 31u, cnt = (uint32_t)m >> 5;
        t->meta_run[m] = (m == 0xFF || off + cnt > 32) ? 0u : (cnt ? ((0xFFFFFFFFu >> (32 - cnt)) << off) : 0u);
    }
    __syncthreads();
}

// A mask of `width` bits starting at bit `start` (mod 32) in one
// instruction; the start's bits above bit 4 are ignored.
__device__ __forceinline__ uint32_t bit_mask_wrap(uint32_t start, uint32_t width) {
    uint32_t r;
    asm("bmsk.wrap.b32 %0, %1, %2;" : "=r"(r) : "r"(start), "r"(width));
    return r;
}

// A mask of `width` bits starting at bit `start` in one instruction (PTX
// bmsk): a leaf's triangle bits.  width 0 (an empty slot) gives 0.
__device__ __forceinline__ uint32_t bit_mask(uint32_t start, uint32_t width) {
    uint32_t r;
    asm("bmsk.clamp.b32 %0, %1, %2;" : "=r"(r) : "r"(start), "r"(width));
    return r;
}

// Stack of node groups: x = child base, y = hit mask (8 bits, near-to-far
// order) | inner mask << 8 | flags << 16.  The top SS entries sit in shared
// memory (one column per thread of a T-thread CTA), the rest of the
// RTB_STACK_TOTAL entries in local memory.
template <int T, int SS>
struct WalkT {
    // shared entries used: SS, or fewer when the whole stack is smaller
    static constexpr int S = SS < RTB_STACK_TOTAL ? SS : RTB_STACK_TOTAL - 1;
    static constexpr int L = RTB_STACK_TOTAL - S;
    uint2 ng;
    int sp;
    int sb;  // entries below sb were handed to helper lanes (RTB_HELPERS); 0 otherwise
    __device__ __forceinline__ void start() { sp = 0; sb = 0; }
    __device__ __forceinline__ bool push(uint2 e, uint2 (*ss)[T], uint2* ls) {
        if (sp < S) ss[sp][threadIdx.x] = e;
        else if (sp < S + L) ls[sp - S] = e;
        else return false;
        sp++;
        return true;
    }
    __device__ __forceinline__ uint2 pop(uint2 (*ss)[T], uint2* ls) {
        sp--;
        return sp < S ? ss[sp][threadIdx.x] : ls[sp - S];
    }
};
using Walk = WalkT<TRACE_T, SSTACK>;

// Byte k of w as an exact float.  Written as a plain shift, mask and
// conversion, which measured +3 % (closest hit) and +5 % (any hit) over
// building the float 2^23 + byte with a byte permute and subtracting 2^23:
// the conversion runs on the XU pipe and takes load off the integer ALU
// pipe, which bounded the node test (ALU 62 -> 53 %, XU 11 -> 61 % of peak).
__device__ __forceinline__ float qbyte(uint32_t w, int k) { return (float)((w >> (8 * k)) & 0xFFu); }
// The same value by the other route: a byte permute builds the float
// 2^23 + byte and a subtraction removes 2^23 (integer ALU + FMA pipes).
__device__ __forceinline__ float qbyte_p(uint32_t w, int k) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, (uint32_t)k | 0x7540u)) - 8388608.0f;
}
// How many of a child's six planes take the byte-permute route (the rest
// convert on the XU pipe), spreading the decode over both pipes: 2 measured
// +1 % over 0 on closest and any hit; 1 and 3 in between.
#ifndef RTB_PRMT_PLANES
#define RTB_PRMT_PLANES 2
#endif
// RTB_PACK_CLOSEST / RTB_PACK_ANY: the node test of the single-level
// closest-hit / any-hit kernel computes a child's near and far plane of one
// axis with one packed f32x2 FMA (sm_100's FFMA2; each component is the same
// round-to-nearest FMA, so the box test and every result are unchanged), and
// removes the 2^23 bias of the two byte-permuted z planes with one packed
// add.  The x and y planes convert on the XU pipe, the z planes by byte
// permute.  Measured on 2M incoherent rays (three alternating runs, results
// byte-identical): closest hit +1.5 %, any hit -0.7 % (left off); packing
// slots k and k + 4 instead: -0.7 % / -0.3 %; all planes converted on the
// XU pipe: -1.9 % / -5.4 %; y planes byte-permuted too: -1.3 % / -1.8 %.
#ifndef RTB_PACK_CLOSEST
#define RTB_PACK_CLOSEST 1
#endif
#ifndef RTB_PACK_ANY
#define RTB_PACK_ANY 0
#endif
// Byte k of w as the exact float 2^15 + byte, built by one byte permute:
// bits 0x47 00 qq 00 are exponent 142 and mantissa q << 8, i.e.
// 2^15 (1 + q 2^-15).  The node test folds the 2^15 bias into its offsets
// (RTB_DECODE15), so a plane costs one integer op and its FMA.
__device__ __forceinline__ float qbyte15(uint32_t w, int k) {
    return __uint_as_float(__byte_perm(w, 0x47000000u, 0x7604u | ((uint32_t)k << 4)));
}
#ifndef RTB_DECODE15
#define RTB_DECODE15 0
#endif
#if RTB_DECODE15
#define RTB_QB(w, k, plane) qbyte15((w), (k))
#else
#define RTB_QB(w, k, plane) ((plane) < RTB_PRMT_PLANES ? qbyte_p((w), (k)) : qbyte((w), (k)))
#endif

// Pulls the node a group will visit next toward L1 (80-byte nodes may span
// two 128-byte lines).
__device__ __forceinline__ void prefetch_next(const uint4* nodes, uint2 ng, uint32_t oct) {
#if RTB_PREFETCH
    const uint32_t h = ng.y & 0xFFu;
    if (h) {
        const uint32_t slot = (uint32_t)(__ffs(h) - 1) ^ oct;
        const uint32_t ni = ng.x + __popc(((ng.y >> 8) & 0xFFu) & ((1u << slot) - 1));
        const char* p = reinterpret_cast<const char*>(nodes + (size_t)ni * 5);
        asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(p + 79));
    }
#else
    (void)nodes; (void)ng; (void)oct;
#endif
}

// Fetches one 8-wide node and tests its eight child boxes against the ray
// segment [tmin, thit].  Outputs the node group of hit inner children
// (`ng`), and the triangle base + 32-bit mask of hit leaf triangles.
// PACK: plane distances by packed f32x2 FMAs (RTB_PACK_CLOSEST).
template <int SLOT = RTB_SLOTMASK, bool PACK = false>
__device__ __forceinline__ void visit_node(const uint4* __restrict__ np, const Ray& r, float thit,
                                           uint32_t& inner_hits, uint32_t& tri_base, uint32_t& tmask, uint2& ng,
                                           const NodeLuts* __restrict__ luts = nullptr) {
    const uint4 w0 = ld_node(np), w1 = ld_node(np + 1), w2 = ld_node(np + 2), w3 = ld_node(np + 3),
                w4 = ld_node(np + 4);
    const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
    const uint32_t e = w0.w;
    const float sx = __uint_as_float((e & 0xFFu) << 23);
    const float sy = __uint_as_float(((e >> 8) & 0xFFu) << 23);
    const float sz = __uint_as_float(((e >> 16) & 0xFFu) << 23);
    const uint32_t imask = e >> 24;
    // per axis: S = s/d, O = (p - o)/d, slack E = 2^-22 |O|
    const float Sx = sx * r.ix, Sy = sy * r.iy, Sz = sz * r.iz;
    const float Ox = (px - r.ox) * r.ix, Oy = (py - r.oy) * r.iy, Oz = (pz - r.oz) * r.iz;
#if RTB_DECODE15
    // planes decode to 2^15 + q, so the offsets carry -B = -2^15 S (exact:
    // a power-of-two scaling).  C = O - B is rounded once, by at most
    // 2^-24 (|O| + |B|), and C -+ E once more; the slack
    // E = 2^-21 |O| + 2^-22 |B| covers both roundings and the error of O
    // itself with a factor of two to spare, so the test stays conservative.
    const float Bx = Sx * 32768.f, By = Sy * 32768.f, Bz = Sz * 32768.f;
    const float Cx = Ox - Bx, Cy = Oy - By, Cz = Oz - Bz;
    const float Ex = fmaf(fabsf(Bx), 0x1p-22f, fabsf(Ox) * 0x1p-21f);
    const float Ey = fmaf(fabsf(By), 0x1p-22f, fabsf(Oy) * 0x1p-21f);
    const float Ez = fmaf(fabsf(Bz), 0x1p-22f, fabsf(Oz) * 0x1p-21f);
    const float Onx = Cx - Ex, Ofx = Cx + Ex, Ony = Cy - Ey, Ofy = Cy + Ey, Onz = Cz - Ez, Ofz = Cz + Ez;
#else
    const float Onx = fmaf(-fabsf(Ox), 0x1p-22f, Ox), Ofx = fmaf(fabsf(Ox), 0x1p-22f, Ox);
    const float Ony = fmaf(-fabsf(Oy), 0x1p-22f, Oy), Ofy = fmaf(fabsf(Oy), 0x1p-22f, Oy);
    const float Onz = fmaf(-fabsf(Oz), 0x1p-22f, Oz), Ofz = fmaf(fabsf(Oz), 0x1p-22f, Oz);
#endif
    // near plane = lo for a positive 1/d, hi otherwise
    const bool nx = r.oct & 1u, ny = r.oct & 2u, nz = r.oct & 4u;
    const uint32_t qnx0 = nx ? w2.z : w2.x, qnx1 = nx ? w2.w : w2.y, qfx0 = nx ? w2.x : w2.z, qfx1 = nx ? w2.y : w2.w;
    const uint32_t qny0 = ny ? w3.z : w3.x, qny1 = ny ? w3.w : w3.y, qfy0 = ny ? w3.x : w3.z, qfy1 = ny ? w3.y : w3.w;
    const uint32_t qnz0 = nz ? w4.z : w4.x, qnz1 = nz ? w4.w : w4.y, qfz0 = nz ? w4.x : w4.z, qfz1 = nz ? w4.y : w4.w;
    uint32_t nh = 0, th = 0;
    uint32_t hm = 0;  // SLOT != 0: hit children in slot order
    // slot s given its six plane distances: the hit test and its bookkeeping
    auto slot = [&](int s, float tnx, float tfx, float tny, float tfy, float tnz, float tfz) {
        const int sh = (s & 3) * 8;
        const float tn = max3f(tnx, tny, fmaxf(tnz, r.tmin));
        const float tf = min3f(tfx, tfy, fminf(tfz, thit));
        const bool hit = tn <= fmaf(fabsf(tf), 0x1p-21f, tf);
        if (SLOT == 1) {
            // leaf run from the meta byte (count << 5 | offset); inner slots
            // (meta 0xFF) are excluded by the inner bit, empty slots have count 0
            const uint32_t mw = s < 4 ? w1.z : w1.w;
            const uint32_t run = bit_mask_wrap(mw >> sh, (mw >> (sh + 5)) & 7u);
            if (hit) hm |= 1u << s;
            if (hit && !((imask >> s) & 1u)) th |= run;
            return;
        }
        if (SLOT == 2) {
            const uint32_t mw = s < 4 ? w1.z : w1.w;
            if (hit) {
                hm |= 1u << s;
                th |= luts->meta_run[(mw >> sh) & 0xFFu];
            }
            return;
        }
        const uint32_t meta = ((s < 4 ? w1.z : w1.w) >> sh) & 0xFFu;
#if RTB_BRANCHLESS
        const uint32_t inner = (imask >> s) & 1u;
        const uint32_t hb = hit ? 1u : 0u;
        nh |= (hb & inner) << ((uint32_t)s ^ r.oct);
        th |= bit_mask(meta & 31u, meta >> 5) & (0u - (hb & (inner ^ 1u)));
#else
        if (hit) {
            if ((imask >> s) & 1u) {
                nh |= 1u << ((uint32_t)s ^ r.oct);
            } else {
                th |= bit_mask(meta & 31u, meta >> 5);  // empty slot: meta 0, no bits
            }
        }
#endif
    };
    if (PACK) {
        const float2 S2x = make_float2(Sx, Sx), S2y = make_float2(Sy, Sy), S2z = make_float2(Sz, Sz);
        const float2 O2x = make_float2(Onx, Ofx), O2y = make_float2(Ony, Ofy), O2z = make_float2(Onz, Ofz);
        const float2 bias = make_float2(-8388608.0f, -8388608.0f);
#pragma unroll
        for (int s = 0; s < 8; s++) {
            const uint32_t k = (uint32_t)s & 3u;
            const uint32_t bx0 = s < 4 ? qnx0 : qnx1, bx1 = s < 4 ? qfx0 : qfx1;
            const uint32_t by0 = s < 4 ? qny0 : qny1, by1 = s < 4 ? qfy0 : qfy1;
            const uint32_t bz0 = s < 4 ? qnz0 : qnz1, bz1 = s < 4 ? qfz0 : qfz1;
            // (near, far) of each axis; z planes as 2^23 + q, less 2^23 (exact)
            const float2 qz = __fadd2_rn(make_float2(__uint_as_float(__byte_perm(bz0, 0x4B000000u, k | 0x7540u)),
                                                     __uint_as_float(__byte_perm(bz1, 0x4B000000u, k | 0x7540u))),
                                         bias);
            const float2 tx = __ffma2_rn(make_float2(qbyte(bx0, (int)k), qbyte(bx1, (int)k)), S2x, O2x);
            const float2 ty = __ffma2_rn(make_float2(qbyte(by0, (int)k), qbyte(by1, (int)k)), S2y, O2y);
            const float2 tz = __ffma2_rn(qz, S2z, O2z);
            slot(s, tx.x, tx.y, ty.x, ty.y, tz.x, tz.y);
        }
    } else {
#pragma unroll
        for (int s = 0; s < 8; s++) {
            const uint32_t bx0 = s < 4 ? qnx0 : qnx1, bx1 = s < 4 ? qfx0 : qfx1;
            const uint32_t by0 = s < 4 ? qny0 : qny1, by1 = s < 4 ? qfy0 : qfy1;
            const uint32_t bz0 = s < 4 ? qnz0 : qnz1, bz1 = s < 4 ? qfz0 : qfz1;
            slot(s, fmaf(RTB_QB(bx0, s & 3, 5), Sx, Onx), fmaf(RTB_QB(bx1, s & 3, 4), Sx, Ofx),
                 fmaf(RTB_QB(by0, s & 3, 3), Sy, Ony), fmaf(RTB_QB(by1, s & 3, 2), Sy, Ofy),
                 fmaf(RTB_QB(bz0, s & 3, 1), Sz, Onz), fmaf(RTB_QB(bz1, s & 3, 0), Sz, Ofz));
        }
    }
    if (SLOT) nh = luts->oct_perm[(r.oct << 8) | (hm & imask)];
    inner_hits = nh;
    tri_base = w1.y;
    tmask = th;
    ng = make_uint2(w1.x, nh | (imask << 8));
}

}  // namespace rtb
