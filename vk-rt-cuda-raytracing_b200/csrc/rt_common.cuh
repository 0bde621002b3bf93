// rt_common.cuh -- shared device types and arithmetic for the B200 ray
// traversal engine.
//
// Layout in HBM (all 16-byte aligned, fetched with 16-byte vector loads):
//   Bvh8Node  80 B  five uint4 words (see below): an 8-wide node whose child
//                   boxes are quantised to 8 bits per plane relative to the
//                   node origin p with a power-of-two scale per axis.
//   TriRec    48 B  three float4: (v0, prim id bits), (e1 = v1-v0, 0), (e2 = v2-v0, 0)
//   RtRay     32 B  (org, tmin), (dir, tmax)
//   RtHit     16 B  (t, prim, u, v)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/rt_b200.h"

namespace rtb {

constexpr int kMaxLeafTris = 7;      // leaf meta holds count-1 in 3 bits
constexpr int kNodeTriSlots = 32;    // triangles referenced by one node
constexpr int kBins = 32;            // SAH bins per axis

// --------------------------------------------------------------------------
// Bvh8Node word layout
//   w0: p.x, p.y, p.z (float bits), {ex, ey, ez, imask} (bytes, little end.)
//   w1: child_base, tri_base, meta[0..3], meta[4..7]
//   w2: qlo.x[0..7], qhi.x[0..7]        (8 bytes each)
//   w3: qlo.y[0..7], qhi.y[0..7]
//   w4: qlo.z[0..7], qhi.z[0..7]
// Scale of axis a is 2^(e_a - 127) (the float whose exponent field is e_a;
// e_a == 0 gives scale 0 for a flat axis).  Child slot i:
//   internal  imask bit i set; its node index is
//             child_base + popc(imask & ((1 << i) - 1))
//   leaf      imask bit i clear, meta[i] = (count << 5) | offset, count 1..7,
//             triangles tri_base + offset .. + count - 1
//   empty     imask bit i clear, meta[i] == 0
// Slots are assigned per node so that slot s holds the child nearest along
// the direction whose sign bits are s; a ray of octant o visits slot k ^ o
// for k = 0, 1, ... (near to far).
// --------------------------------------------------------------------------
struct __align__(16) Bvh8Node {
    uint4 w[5];
};
static_assert(sizeof(Bvh8Node) == 80, "Bvh8Node is 80 bytes");

struct __align__(16) TriRec {
    float4 a;  // v0.xyz, prim id (int bits)
    float4 b;  // e1.xyz, 0
    float4 c;  // e2.xyz, 0
};
static_assert(sizeof(TriRec) == 48, "TriRec is 48 bytes");

// Binary BVH produced by the SAH builder (intermediate + source of the
// stackless/BVH4 exports).  Inner: a = left, b = right.  Leaf: a = first
// position in the primitive permutation, b = -count.
struct __align__(16) Node2 {
    float lo[3];
    int a;
    float hi[3];
    int b;
};
static_assert(sizeof(Node2) == 32, "Node2 is 32 bytes");

// --------------------------------------------------------------------------
// Exact-rounding arithmetic.  The triangle test below spells every operation
// with an _rn intrinsic so nvcc never contracts it into an FMA; the CPU
// oracle evaluates the same expression tree with -ffp-contract=off, which
// makes t, u, v and the accepted primitive bit-identical.
// --------------------------------------------------------------------------
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

// Moller-Trumbore as in layer/cuda_bvh_backend.cu:143-157 (|det| < 1e-12
// rejects, inclusive barycentric bounds).  Returns false on rejection; the
// caller applies the (tmin, tmax) interval and the tie rule.
__device__ __forceinline__ bool intersect_tri(float ox, float oy, float oz, float dx, float dy, float dz,
                                              const float4& A, const float4& B, const float4& Cc,
                                              float& t, float& u, float& v) {
    const float e1x = B.x, e1y = B.y, e1z = B.z;
    const float e2x = Cc.x, e2y = Cc.y, e2z = Cc.z;
    const float px = sub(mul(dy, e2z), mul(dz, e2y));
    const float py = sub(mul(dz, e2x), mul(dx, e2z));
    const float pz = sub(mul(dx, e2y), mul(dy, e2x));
    const float det = add(add(mul(e1x, px), mul(e1y, py)), mul(e1z, pz));
    if (fabsf(det) < 1e-12f) return false;
    const float inv = __frcp_rn(det);  // correctly rounded 1/det, as 1.f/det
    const float sx = sub(ox, A.x), sy = sub(oy, A.y), sz = sub(oz, A.z);
    u = mul(inv, add(add(mul(sx, px), mul(sy, py)), mul(sz, pz)));
    if (u < 0.f || u > 1.f) return false;
    const float qx = sub(mul(sy, e1z), mul(sz, e1y));
    const float qy = sub(mul(sz, e1x), mul(sx, e1z));
    const float qz = sub(mul(sx, e1y), mul(sy, e1x));
    v = mul(inv, add(add(mul(dx, qx), mul(dy, qy)), mul(dz, qz)));
    if (v < 0.f || add(u, v) > 1.f) return false;
    t = mul(inv, add(add(mul(e2x, qx), mul(e2y, qy)), mul(e2z, qz)));
    return true;
}

// Instance ray transform (inverse 3x4, row major), layer/rt_ir_exec.cu:81-91:
// left-to-right sums, no contraction, direction left unnormalised.
__device__ __forceinline__ void xform_point(const float* m, float x, float y, float z, float& ox, float& oy,
                                            float& oz) {
    ox = add(add(add(mul(m[0], x), mul(m[1], y)), mul(m[2], z)), m[3]);
    oy = add(add(add(mul(m[4], x), mul(m[5], y)), mul(m[6], z)), m[7]);
    oz = add(add(add(mul(m[8], x), mul(m[9], y)), mul(m[10], z)), m[11]);
}
__device__ __forceinline__ void xform_dir(const float* m, float x, float y, float z, float& ox, float& oy,
                                          float& oz) {
    ox = add(add(mul(m[0], x), mul(m[1], y)), mul(m[2], z));
    oy = add(add(mul(m[4], x), mul(m[5], y)), mul(m[6], z));
    oz = add(add(mul(m[8], x), mul(m[9], y)), mul(m[10], z));
}

// --------------------------------------------------------------------------
// Float <-> order-preserving uint (for atomicMin/atomicMax on floats).
// --------------------------------------------------------------------------
__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// --------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11) -- same stream as the host/oracle.
// --------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}
__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

// Byte b (0..7) of a 64-bit pair (lo word, hi word) as an exact float.
__device__ __forceinline__ float byte_f(uint32_t lo, uint32_t hi, int b) {
    const uint32_t w = b < 4 ? lo : hi;
    return (float)((w >> ((b & 3) * 8)) & 0xFFu);
}

}  // namespace rtb
