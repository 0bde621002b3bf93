// rt_trace.cu -- closest-hit and any-hit traversal of the compressed 8-wide
// BVH (replaces bk_tracePrimaryDense / bk_traceDiffuseArbitrary,
// layer/cuda_bvh_backend.cu:104-183,526-598, and the any-hit traceShadow,
// v10_pipeline.cu:195-251).
//
// Execution model (B200, 148 SMs): persistent warps sized to fill every SM;
// each lane owns one ray; idle lanes refill from a global ray counter with
// one warp-aggregated atomic (dynamic fetch), so warps stay full while ray
// lengths diverge.  Per node: one 80-byte node = five 16-byte loads; the
// eight child boxes are decoded from 8-bit planes with one FMA per plane
// and tested against the ray; hit inner children become an 8-bit mask in
// near-to-far order (slot ^ octant), hit leaves a 32-bit triangle mask.  The
// traversal stack holds (child base, hit mask, inner mask) groups: the top
// SSTACK entries live in shared memory, the rest in local memory; overflow
// is reported through the status word, never dropped.
//
// Box test robustness: t = q * (s/d) + (p - o)/d is evaluated with an
// absolute slack of 2^-22 |(p - o)/d| folded into the near/far offsets and
// a relative slack of 2^-21 on the far distance, which bounds every
// rounding of the decode, so a box that contains an accepted triangle hit
// is never culled.  Hit results are therefore defined by the triangle test
// alone: Moller-Trumbore in exact IEEE single precision (rt_common.cuh),
// ties on t resolved toward the lower primitive id.
#include <cfloat>

#include "rt_internal.h"
#include "rt_trace.cuh"

namespace rtb {

template <bool ANY, bool COUNT>
__global__ void __launch_bounds__(TRACE_T, TRACE_MINB)
    k_trace_blas(const uint4* __restrict__ nodes, const float4* __restrict__ tris, const RtRay* __restrict__ rays,
                 int n, RtHit* __restrict__ hits, uint8_t* __restrict__ occ, uint32_t* __restrict__ counts,
                 int* __restrict__ work, int* __restrict__ status) {
    __shared__ uint2 sstack[SSTACK][TRACE_T];
    uint2 lstack[LSTACK];
    const int lane = threadIdx.x & 31;
    int ray = -1;
    bool exhausted = false;
    Ray r;
    Walk w;
    float thit = 0.f, hu = 0.f, hv = 0.f;
    int hprim = -1;
    uint32_t cn = 0, ct = 0;
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
                    r = load_ray(rays, ri);
                    thit = r.tmax;
                    hprim = -1;
                    hu = hv = 0.f;
                    w.start();
                    w.ng = make_uint2(0u, (1u << r.oct) | (1u << 8));
                    cn = ct = 0;
                } else {
                    exhausted = true;
                }
            }
        }
        if (__all_sync(FULL_MASK, ray < 0)) break;
        if (ray < 0) continue;
        // ---- one node visit ----
        uint32_t tri_base = 0, tmask = 0;
        if (w.ng.y & 0xFFu) {
            uint32_t hitsm = w.ng.y & 0xFFu;
            const uint32_t imask = (w.ng.y >> 8) & 0xFFu;
            const int k = __ffs(hitsm) - 1;
            hitsm &= hitsm - 1;
            const uint32_t slot = (uint32_t)k ^ r.oct;
            const uint32_t ni = w.ng.x + __popc(imask & ((1u << slot) - 1));
            if (hitsm) {
                if (!w.push(make_uint2(w.ng.x, hitsm | (imask << 8)), sstack, lstack)) {
                    atomicOr(status, RT_STATUS_STACK);
                    hprim = -2;
                    goto finish;
                }
            }
            if (COUNT) cn++;
            uint32_t nmask;
            visit_node(nodes + (size_t)ni * 5, r, thit, nmask, tri_base, tmask, w.ng);
            (void)nmask;
        }
        // ---- triangles of the node just visited ----
        while (tmask) {
            const int j = __ffs(tmask) - 1;
            tmask &= tmask - 1;
            const float4* tp = tris + (size_t)(tri_base + j) * 3;
            const float4 A = __ldg(tp), B = __ldg(tp + 1), Cc = __ldg(tp + 2);
            if (COUNT) ct++;
            float t, u, v;
            if (intersect_tri(r.ox, r.oy, r.oz, r.dx, r.dy, r.dz, A, B, Cc, t, u, v)) {
                const int prim = __float_as_int(A.w);
                if (ANY) {
                    if (t > r.tmin && t < r.tmax) {
                        hprim = prim;
                        goto finish;
                    }
                } else if (t > r.tmin && (t < thit || (t == thit && hprim >= 0 && prim < hprim))) {
                    thit = t;
                    hprim = prim;
                    hu = u;
                    hv = v;
                }
            }
        }
        if ((w.ng.y & 0xFFu) == 0) {
            if (w.sp == 0) goto finish;
            w.ng = w.pop(sstack, lstack);
        }
        continue;
    finish:
        if (ANY) {
            occ[ray] = hprim >= 0 ? 1 : 0;
        } else {
            RtHit h;
            h.t = hprim >= 0 ? thit : __int_as_float(0x7f800000);
            h.prim = hprim >= 0 ? hprim : -1;
            h.u = hprim >= 0 ? hu : 0.f;
            h.v = hprim >= 0 ? hv : 0.f;
            reinterpret_cast<float4*>(hits)[ray] = make_float4(h.t, __int_as_float(h.prim), h.u, h.v);
        }
        if (COUNT) reinterpret_cast<uint2*>(counts)[ray] = make_uint2(cn, ct);
        ray = -1;
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

int launch_trace_blas(const Bvh8Device& b, const RtRay* rays, int n, RtHit* hits, uint8_t* occ,
                      uint32_t* counts, int* work, int* status, cudaStream_t s) {
    const uint4* nodes = reinterpret_cast<const uint4*>(b.nodes.p);
    const float4* tris = reinterpret_cast<const float4*>(b.tris.p);
    if (counts) {
        if (occ) {
            static const int g = persistent_grid(k_trace_blas<true, true>, TRACE_T);
            k_trace_blas<true, true><<<g, TRACE_T, 0, s>>>(nodes, tris, rays, n, hits, occ, counts, work, status);
        } else {
            static const int g = persistent_grid(k_trace_blas<false, true>, TRACE_T);
            k_trace_blas<false, true><<<g, TRACE_T, 0, s>>>(nodes, tris, rays, n, hits, occ, counts, work, status);
        }
    } else if (occ) {
        static const int g = persistent_grid(k_trace_blas<true, false>, TRACE_T);
        k_trace_blas<true, false><<<g, TRACE_T, 0, s>>>(nodes, tris, rays, n, hits, occ, counts, work, status);
    } else {
        static const int g = persistent_grid(k_trace_blas<false, false>, TRACE_T);
        k_trace_blas<false, false><<<g, TRACE_T, 0, s>>>(nodes, tris, rays, n, hits, occ, counts, work, status);
    }
    return cudaGetLastError() == cudaSuccess ? RT_OK : RT_ERR_CUDA;
}

}  // namespace rtb
