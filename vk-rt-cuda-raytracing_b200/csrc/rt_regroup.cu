// rt_regroup.cu -- ray regrouping for coherence: rtRays_regroup.
//
// The reference sorts ray batches by the 30-bit Morton code of their
// origins before tracing: on the GPU with CUB's radix sort in its benchmark
// (cuda_rt_v40.cu:94-124, 1226-1239) and with a 4-pass radix sort on the host
// inside its per-call trace path (layer/cuda_bvh_backend.cu:1387-1433).  Rays
// next to each other in a warp then start in the same part of the tree.
//
// Here: a key per ray (the reference's origin Morton code, or the direction
// octant above a 29-bit Morton code, optionally cut to its top 16 bits),
// then this file's own stable LSD radix sort on the device, 8 bits per pass
// (2 passes for 16-bit keys, 4 for 32): per tile a digit histogram, one
// exclusive scan over (digit, tile) counts for every tile's output offsets,
// and a scatter that ranks equal digits in tile order (warp __match_any_sync
// peers plus per-warp digit counts in shared memory, round by round), so
// equal keys keep their input order.  Rays and an optional payload of one
// int per ray (the path tracer's path ids) are gathered once at the end.
// The ray count may come from device memory (a queue length written by an
// earlier kernel); every launch is sized for the capacity.
#include <algorithm>

#include "rt_internal.h"

namespace rtb {

constexpr int RG_T = 256;                 // threads per block
constexpr int RG_ROUNDS = 8;              // items per thread and tile
constexpr int RG_TILE = RG_T * RG_ROUNDS; // items per tile
constexpr int RG_BINS = 256;

// 10 bits of v spread to every third bit (the standard Morton bit spread).
__device__ __forceinline__ uint32_t spread10(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t quant10(float x, float lo, float inv_ext) {
    const float q = (x - lo) * inv_ext * 1024.0f;
    return (uint32_t)fminf(fmaxf(q, 0.0f), 1023.0f);
}

// kind RT_REGROUP_MORTON: 30-bit Morton code of the origin in the box (the
// reference's key); RT_REGROUP_OCTANT_MORTON: direction octant in bits
// 29-31 above the top 29 bits of that code.  key_bits 16 keeps the top 16.
__global__ void k_rg_keys(const RtRay* __restrict__ rays, int cap, const int* __restrict__ d_n, int n_host,
                          float4 lo, float4 inv_ext, int kind, int key_bits, uint32_t* __restrict__ keys,
                          int* __restrict__ idx) {
    const int n = d_n ? min(*d_n, cap) : n_host;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = __ldg(reinterpret_cast<const float4*>(rays + i));
    const float4 d = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
    const uint32_t m = (spread10(quant10(o.x, lo.x, inv_ext.x)) << 2) | (spread10(quant10(o.y, lo.y, inv_ext.y)) << 1) |
                       spread10(quant10(o.z, lo.z, inv_ext.z));
    uint32_t k = m;
    if (kind == RT_REGROUP_OCTANT_MORTON) {
        const uint32_t oct = (signbit(d.x) ? 4u : 0u) | (signbit(d.y) ? 2u : 0u) | (signbit(d.z) ? 1u : 0u);
        k = (oct << 29) | (m >> 1);
    } else {
        k = m << 2;  // 30 bits at the top
    }
    if (key_bits == 16) k >>= 16;
    keys[i] = k;
    idx[i] = i;
}

// counts[digit * tiles + tile] = items of `tile` whose key has `digit` at bit `shift`.
__global__ void __launch_bounds__(RG_T) k_rg_hist(const uint32_t* __restrict__ keys, int cap,
                                                  const int* __restrict__ d_n, int n_host, int shift, int tiles,
                                                  int* __restrict__ counts) {
    __shared__ int s_hist[RG_BINS];
    const int n = d_n ? min(*d_n, cap) : n_host;
    s_hist[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * RG_TILE;
    for (int j = 0; j < RG_ROUNDS; j++) {
        const int i = base + j * RG_T + threadIdx.x;
        if (i < n) atomicAdd(&s_hist[(keys[i] >> shift) & 0xFFu], 1);
    }
    __syncthreads();
    counts[threadIdx.x * tiles + blockIdx.x] = s_hist[threadIdx.x];
}

// Stable scatter of (key, value) pairs by the digit at `shift`.
__global__ void __launch_bounds__(RG_T) k_rg_scatter(const uint32_t* __restrict__ keys_in,
                                                     const int* __restrict__ vals_in, int cap,
                                                     const int* __restrict__ d_n, int n_host, int shift, int tiles,
                                                     const int* __restrict__ offs, uint32_t* __restrict__ keys_out,
                                                     int* __restrict__ vals_out) {
    __shared__ int s_run[RG_BINS];                // items of each digit placed by earlier rounds
    __shared__ int s_wcnt[RG_T / 32][RG_BINS];    // this round's count per warp and digit
    const int n = d_n ? min(*d_n, cap) : n_host;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    s_run[threadIdx.x] = offs[threadIdx.x * tiles + blockIdx.x];
    for (int w = 0; w < RG_T / 32; w++) s_wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * RG_TILE;
    for (int j = 0; j < RG_ROUNDS; j++) {
        const int i = base + j * RG_T + threadIdx.x;
        const bool live = i < n;
        const uint32_t key = live ? keys_in[i] : 0u;
        const uint32_t dig = live ? (key >> shift) & 0xFFu : RG_BINS;  // a value no live lane has
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, dig);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (live && rank == 0) s_wcnt[warp][dig] = __popc(peers);
        __syncthreads();
        if (live) {
            int pos = s_run[dig] + rank;
            for (int w = 0; w < warp; w++) pos += s_wcnt[w][dig];
            keys_out[pos] = key;
            vals_out[pos] = vals_in[i];
        }
        __syncthreads();
        int add = 0;
        for (int w = 0; w < RG_T / 32; w++) {
            add += s_wcnt[w][threadIdx.x];
            s_wcnt[w][threadIdx.x] = 0;
        }
        s_run[threadIdx.x] += add;
        __syncthreads();
    }
}

__global__ void k_rg_gather(const RtRay* __restrict__ in, const int* __restrict__ pay_in, int cap,
                            const int* __restrict__ d_n, int n_host, const int* __restrict__ idx,
                            RtRay* __restrict__ out, int* __restrict__ pay_out, int32_t* __restrict__ perm) {
    const int n = d_n ? min(*d_n, cap) : n_host;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int s = idx[k];
    const float4* src = reinterpret_cast<const float4*>(in + s);
    float4* dst = reinterpret_cast<float4*>(out + k);
    dst[0] = __ldg(src);
    dst[1] = __ldg(src + 1);
    if (pay_out) pay_out[k] = pay_in[s];
    if (perm) perm[k] = s;
}

// Shared by rtRays_regroup and the path tracer: sorts rays[0 .. n) (n from
// d_n when given, at most cap) into out (and the payload alongside).
bool regroup_rays(const RtRay* rays, const int* payload, int cap, const int* d_n, int n_host, const float* box6,
                  int kind, int key_bits, RtRay* out, int* payload_out, int32_t* perm, cudaStream_t s) {
    if (cap <= 0) return true;
    const int tiles = (cap + RG_TILE - 1) / RG_TILE;
    TmpBuf<uint32_t> keys;
    TmpBuf<int> vals, counts, offs;
    if (!keys.alloc((size_t)cap * 2, s) || !vals.alloc((size_t)cap * 2, s) ||
        !counts.alloc((size_t)RG_BINS * tiles, s) || !offs.alloc((size_t)RG_BINS * tiles, s))
        return false;
    float4 lo = make_float4(box6[0], box6[1], box6[2], 0.f), ie;
    ie.x = box6[3] > box6[0] ? 1.0f / (box6[3] - box6[0]) : 0.f;
    ie.y = box6[4] > box6[1] ? 1.0f / (box6[4] - box6[1]) : 0.f;
    ie.z = box6[5] > box6[2] ? 1.0f / (box6[5] - box6[2]) : 0.f;
    ie.w = 0.f;
    const int blocks = (cap + 255) / 256;
    uint32_t* k0 = keys.p;
    uint32_t* k1 = keys.p + cap;
    int* v0 = vals.p;
    int* v1 = vals.p + cap;
    k_rg_keys<<<blocks, 256, 0, s>>>(rays, cap, d_n, n_host, lo, ie, kind, key_bits, k0, v0);
    for (int shift = 0; shift < key_bits; shift += 8) {
        k_rg_hist<<<tiles, RG_T, 0, s>>>(k0, cap, d_n, n_host, shift, tiles, counts.p);
        if (!scan_exclusive(counts.p, offs.p, RG_BINS * tiles, nullptr, s)) return false;
        k_rg_scatter<<<tiles, RG_T, 0, s>>>(k0, v0, cap, d_n, n_host, shift, tiles, offs.p, k1, v1);
        std::swap(k0, k1);
        std::swap(v0, v1);
    }
    k_rg_gather<<<blocks, 256, 0, s>>>(rays, payload, cap, d_n, n_host, v0, out, payload_out, perm);
    return RT_CUDA(cudaGetLastError());
}

}  // namespace rtb

using namespace rtb;

extern "C" int rtRays_regroup(const RtRay* d_in, int n, const float* box6, int kind, int key_bits, RtRay* d_out,
                              int32_t* d_perm, void* stream) {
    if (n < 0 || (n > 0 && (!d_in || !d_out || !box6)) || d_in == d_out ||
        (kind != RT_REGROUP_MORTON && kind != RT_REGROUP_OCTANT_MORTON) || (key_bits != 16 && key_bits != 32)) {
        set_error("rtRays_regroup: invalid argument");
        return RT_ERR_INVALID;
    }
    if (misaligned(d_in, 16) || misaligned(d_out, 16) || misaligned(d_perm, 4)) {
        set_error("rtRays_regroup: rays must be 16-byte aligned, d_perm 4-byte");
        return RT_ERR_INVALID;
    }
    if (n == 0) return RT_OK;
    return regroup_rays(d_in, nullptr, n, nullptr, n, box6, kind, key_bits, d_out, nullptr, d_perm,
                        (cudaStream_t)stream)
               ? RT_OK
               : RT_ERR_CUDA;
}
