// rt_raygen.cu -- next-bounce ray batches made on the device from a
// closest-hit batch: cudaBVH_generateRays.
//
// Replaces the reference's genAndCompact (multi_bounce.cu:281-362) and the
// host-side ray preparation of its benchmarks: for every ray with a hit, the
// hit point p = o + t d, the geometric normal of the hit triangle turned to
// face the ray, then either a cosine-weighted diffuse bounce or a shadow ray
// toward a square area light, with the origin pushed eps along the normal
// (multi_bounce.cu:355-356).  Rays that missed produce nothing: survivors
// are compacted with a warp ballot + popcount and a block scan over the warp
// totals (the scheme of warp_compact.cuh:23-80), but with block offsets
// from an exclusive scan of the block counts instead of an atomic per block,
// so the output order is the input order of the hits and the result is
// deterministic.
//
// Deliberate differences from the reference, all so that the CPU oracle can
// reproduce every output bit: each operation is an explicitly rounded
// single-precision op (no FMA contraction); 1/sqrt is a correctly rounded
// square root and division (reference: rsqrtf); the cosine-weighted
// direction uses Malley's method on a rejection-sampled unit disk (no sin/
// cos; reference: sqrt(1 - r1), 2 pi r2 and __sinf/__cosf); random numbers
// are Philox4x32-10 keyed by (seed, 3) for diffuse and (seed, 4) for shadow
// rays with counter (output index, block, 0, 0) (reference: PCG).
#include <algorithm>

#include "rt_internal.h"

namespace rtb {

constexpr int GEN_T = 256;

__device__ __forceinline__ float rn_sqrt(float x) { return __fsqrt_rn(x); }
__device__ __forceinline__ float rn_div(float a, float b) { return __fdiv_rn(a, b); }

// Uniform [0, 1) floats k*4 .. k*4+3 of output `item` in stream (seed, key1).
__device__ __forceinline__ float4 gen_u4(uint32_t seed, uint32_t key1, uint32_t item, uint32_t block) {
    const uint4 b = philox(make_uint4(item, block, 0u, 0u), make_uint2(seed, key1));
    return make_float4(u01(b.x), u01(b.y), u01(b.z), u01(b.w));
}

// The ray for output `item` leaving the hit of input ray `src`.
__device__ void gen_one(const RtRay* __restrict__ rays, const RtHit* __restrict__ hits,
                        const float* __restrict__ tris9, int src, uint32_t item, const RtRayGen& g,
                        RtRay* __restrict__ out) {
    const float4 ro = __ldg(reinterpret_cast<const float4*>(rays + src));
    const float4 rd = __ldg(reinterpret_cast<const float4*>(rays + src) + 1);
    const RtHit h = hits[src];
    const float px = add(ro.x, mul(h.t, rd.x)), py = add(ro.y, mul(h.t, rd.y)), pz = add(ro.z, mul(h.t, rd.z));
    const float* v = tris9 + (size_t)h.prim * 9;
    const float e1x = sub(v[3], v[0]), e1y = sub(v[4], v[1]), e1z = sub(v[5], v[2]);
    const float e2x = sub(v[6], v[0]), e2y = sub(v[7], v[1]), e2z = sub(v[8], v[2]);
    float nx = sub(mul(e1y, e2z), mul(e1z, e2y));
    float ny = sub(mul(e1z, e2x), mul(e1x, e2z));
    float nz = sub(mul(e1x, e2y), mul(e1y, e2x));
    const float nl = rn_div(1.0f, rn_sqrt(fmaxf(add(add(mul(nx, nx), mul(ny, ny)), mul(nz, nz)), 1e-30f)));
    nx = mul(nx, nl);
    ny = mul(ny, nl);
    nz = mul(nz, nl);
    if (add(add(mul(nx, rd.x), mul(ny, rd.y)), mul(nz, rd.z)) > 0.f) {
        nx = -nx;
        ny = -ny;
        nz = -nz;
    }
    const float ox = add(px, mul(g.eps, nx)), oy = add(py, mul(g.eps, ny)), oz = add(pz, mul(g.eps, nz));
    RtRay r;
    r.org[0] = ox;
    r.org[1] = oy;
    r.org[2] = oz;
    if (g.kind == RT_GEN_DIFFUSE) {
        // tangent frame: branch on the larger of |nx|, |ny| (multi_bounce.cu:332-340)
        float tx, ty, tz;
        if (fabsf(nx) > fabsf(ny)) {
            const float il = rn_div(1.0f, rn_sqrt(add(mul(nx, nx), mul(nz, nz))));
            tx = mul(-nz, il);
            ty = 0.f;
            tz = mul(nx, il);
        } else {
            const float il = rn_div(1.0f, rn_sqrt(add(mul(ny, ny), mul(nz, nz))));
            tx = 0.f;
            ty = mul(nz, il);
            tz = mul(-ny, il);
        }
        const float bx = sub(mul(ny, tz), mul(nz, ty));
        const float by = sub(mul(nz, tx), mul(nx, tz));
        const float bz = sub(mul(nx, ty), mul(ny, tx));
        // Malley: the first of 8 uniform points of [-1,1)^2 inside the unit disk
        float x = 0.f, y = 0.f;
        bool found = false;
#pragma unroll 1
        for (uint32_t blk = 0; blk < 4 && !found; blk++) {
            const float4 u = gen_u4(g.seed, 3u, item, blk);
            const float a0 = sub(mul(2.f, u.x), 1.f), b0 = sub(mul(2.f, u.y), 1.f);
            const float a1 = sub(mul(2.f, u.z), 1.f), b1 = sub(mul(2.f, u.w), 1.f);
            if (add(mul(a0, a0), mul(b0, b0)) < 1.f) {
                x = a0;
                y = b0;
                found = true;
            } else if (add(mul(a1, a1), mul(b1, b1)) < 1.f) {
                x = a1;
                y = b1;
                found = true;
            }
        }
        const float z = rn_sqrt(fmaxf(sub(sub(1.f, mul(x, x)), mul(y, y)), 0.f));
        float dx = add(add(mul(x, tx), mul(y, bx)), mul(z, nx));
        float dy = add(add(mul(x, ty), mul(y, by)), mul(z, ny));
        float dz = add(add(mul(x, tz), mul(y, bz)), mul(z, nz));
        const float dl = rn_div(1.0f, rn_sqrt(add(add(mul(dx, dx), mul(dy, dy)), mul(dz, dz))));
        r.dir[0] = mul(dx, dl);
        r.dir[1] = mul(dy, dl);
        r.dir[2] = mul(dz, dl);
        r.tmin = g.tmin;
        r.tmax = g.tmax;
    } else {
        const float4 u = gen_u4(g.seed, 4u, item, 0u);
        const float lx = add(g.light_center[0], mul(sub(u.x, 0.5f), g.light_size));
        const float ly = g.light_center[1];
        const float lz = add(g.light_center[2], mul(sub(u.y, 0.5f), g.light_size));
        const float dx = sub(lx, ox), dy = sub(ly, oy), dz = sub(lz, oz);
        const float dist = rn_sqrt(add(add(mul(dx, dx), mul(dy, dy)), mul(dz, dz)));
        r.dir[0] = rn_div(dx, dist);
        r.dir[1] = rn_div(dy, dist);
        r.dir[2] = rn_div(dz, dist);
        r.tmin = g.tmin;
        r.tmax = mul(dist, 0.9999f);  // stops just short of the light
    }
    *out = r;
}

// Hits among inputs i of this block, and this thread's rank among them:
// ballot + popcount per warp, warp totals scanned in shared memory.
__device__ __forceinline__ int block_rank(bool alive, int* s_warp, int& block_total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xFFFFFFFFu, alive);
    if (lane == 0) s_warp[warp] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < GEN_T / 32; w++) {
        const int c = s_warp[w];
        before += w < warp ? c : 0;
        total += c;
    }
    __syncthreads();
    block_total = total;
    return before + __popc(m & ((1u << lane) - 1u));
}

// A hit counts when its primitive is one of this BVH's triangles (a record
// with any other id is skipped, never followed into the triangle array).
__device__ __forceinline__ bool live_hit(const RtHit* __restrict__ hits, int i, int n, int ntris) {
    if (i >= n) return false;
    const int p = hits[i].prim;
    return p >= 0 && p < ntris;
}

__global__ void __launch_bounds__(GEN_T) k_gen_count(const RtHit* __restrict__ hits, int n, int ntris,
                                                     int* __restrict__ bcnt) {
    __shared__ int s_warp[GEN_T / 32];
    const int i = blockIdx.x * GEN_T + threadIdx.x;
    int total = 0;
    block_rank(live_hit(hits, i, n, ntris), s_warp, total);
    if (threadIdx.x == 0) bcnt[blockIdx.x] = total;
}

// One ray per hit (count == 0): compaction and generation in one pass.
// Otherwise the survivors' input indices are listed for k_gen_cycle.
__global__ void __launch_bounds__(GEN_T) k_gen_compact(const RtRay* __restrict__ rays, const RtHit* __restrict__ hits,
                                                       const float* __restrict__ tris9, int n, int ntris,
                                                       const int* __restrict__ boff, RtRayGen g, int direct,
                                                       RtRay* __restrict__ out, int32_t* __restrict__ src,
                                                       int* __restrict__ survivors) {
    __shared__ int s_warp[GEN_T / 32];
    const int i = blockIdx.x * GEN_T + threadIdx.x;
    const bool alive = live_hit(hits, i, n, ntris);
    int total = 0;
    const int rank = block_rank(alive, s_warp, total);
    if (!alive) return;
    const int k = boff[blockIdx.x] + rank;
    if (direct) {
        gen_one(rays, hits, tris9, i, (uint32_t)k, g, out + k);
        if (src) src[k] = i;
    } else {
        survivors[k] = i;
    }
}

// count rays, output k from the (k mod m)-th hit, m = *d_m hits.
__global__ void __launch_bounds__(GEN_T) k_gen_cycle(const RtRay* __restrict__ rays, const RtHit* __restrict__ hits,
                                                     const float* __restrict__ tris9, const int* __restrict__ survivors,
                                                     const int* __restrict__ d_m, int count, RtRayGen g,
                                                     RtRay* __restrict__ out, int32_t* __restrict__ src,
                                                     int* __restrict__ d_count) {
    const int m = *d_m;
    const int total = m > 0 ? count : 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_count = total;
    for (int k = blockIdx.x * GEN_T + threadIdx.x; k < total; k += gridDim.x * GEN_T) {
        const int s = survivors[k % m];
        gen_one(rays, hits, tris9, s, (uint32_t)k, g, out + k);
        if (src) src[k] = s;
    }
}

}  // namespace rtb

using namespace rtb;

extern "C" int cudaBVH_generateRays(CudaBVH_t bvh, const RtRay* d_rays, const RtHit* d_hits, int n,
                                    const RtRayGen* gen, RtRay* d_out, int32_t* d_src, int* d_count, void* stream) {
    if (!bvh || !gen || !d_count || n < 0 || (n > 0 && (!d_rays || !d_hits || !d_out)) ||
        (gen->kind != RT_GEN_DIFFUSE && gen->kind != RT_GEN_SHADOW) || gen->count < 0) {
        set_error("cudaBVH_generateRays: invalid argument");
        return RT_ERR_INVALID;
    }
    if (misaligned(d_rays, 16) || misaligned(d_hits, 16) || misaligned(d_out, 16) || misaligned(d_src, 4) ||
        misaligned(d_count, 4)) {
        set_error("cudaBVH_generateRays: rays, hits and output must be 16-byte aligned, d_src and d_count 4-byte");
        return RT_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) return RT_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int), s)) ? RT_OK : RT_ERR_CUDA;
    const int blocks = (n + GEN_T - 1) / GEN_T;
    const bool direct = gen->count == 0;
    TmpBuf<int> bcnt, boff, survivors;
    if (!bcnt.alloc(blocks, s) || !boff.alloc(blocks + 1, s) || (!direct && !survivors.alloc(n, s)))
        return RT_ERR_NOMEM;
    k_gen_count<<<blocks, GEN_T, 0, s>>>(d_hits, n, bvh->num_tris, bcnt.p);
    if (!RT_CUDA(cudaGetLastError())) return RT_ERR_CUDA;
    // boff[blocks] receives the number of hits
    if (!scan_exclusive(bcnt.p, boff.p, blocks, boff.p + blocks, s)) return RT_ERR_CUDA;
    k_gen_compact<<<blocks, GEN_T, 0, s>>>(d_rays, d_hits, bvh->tris9.p, n, bvh->num_tris, boff.p, *gen,
                                          direct ? 1 : 0, d_out,
                                          d_src, direct ? nullptr : survivors.p);
    if (!RT_CUDA(cudaGetLastError())) return RT_ERR_CUDA;
    if (direct) {
        if (!RT_CUDA(cudaMemcpyAsync(d_count, boff.p + blocks, sizeof(int), cudaMemcpyDeviceToDevice, s)))
            return RT_ERR_CUDA;
    } else {
        const int grid = std::min((gen->count + GEN_T - 1) / GEN_T, num_sms() * 8);
        k_gen_cycle<<<std::max(grid, 1), GEN_T, 0, s>>>(d_rays, d_hits, bvh->tris9.p, survivors.p, boff.p + blocks,
                                                        gen->count, *gen, d_out, d_src, d_count);
        if (!RT_CUDA(cudaGetLastError())) return RT_ERR_CUDA;
    }
    return RT_OK;
}
