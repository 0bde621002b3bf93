// rt_probe.cu -- read-bandwidth probe for the roofline figures.
//
// The traversal kernels read an 8-wide BVH and triangle records that stay
// resident in the 126 MB L2 on the benchmark scenes, so their bound is L2
// bandwidth as much as HBM bandwidth.  This probe streams a device buffer
// with 16-byte loads cached in L2 only (ld.global.cg), a grid of resident
// CTAs over all SMs, all passes inside one launch (so launch latency does
// not dilute a small buffer's figure), timed with events: a buffer well
// under the L2 size gives the L2 read bandwidth, one far above it the HBM
// read bandwidth.  No clock, power or other device setting is touched.
#include <algorithm>

#include "rt_internal.h"

namespace rtb {

constexpr int PROBE_T = 256;

__global__ void __launch_bounds__(PROBE_T) k_probe_read(const uint4* __restrict__ p, size_t n16, int passes,
                                                        uint32_t* __restrict__ sink) {
    const size_t stride = (size_t)gridDim.x * PROBE_T;
    uint32_t acc = 0;
    for (int pass = 0; pass < passes; pass++) {
        size_t i = (size_t)blockIdx.x * PROBE_T + threadIdx.x;
        // four independent loads in flight per thread
        for (; i + 3 * stride < n16; i += 4 * stride) {
            const uint4 a = __ldcg(p + i), b = __ldcg(p + i + stride), c = __ldcg(p + i + 2 * stride),
                        d = __ldcg(p + i + 3 * stride);
            acc ^= a.x ^ a.y ^ a.z ^ a.w ^ b.x ^ b.y ^ b.z ^ b.w ^ c.x ^ c.y ^ c.z ^ c.w ^ d.x ^ d.y ^ d.z ^ d.w;
        }
        for (; i < n16; i += stride) {
            const uint4 a = __ldcg(p + i);
            acc ^= a.x ^ a.y ^ a.z ^ a.w;
        }
    }
    // the buffer is filled with a pattern whose XOR never equals this value,
    // so the store never happens, but the compiler must keep every load
    if (acc == 0x9E3779B9u) sink[0] = acc;
}

}  // namespace rtb

using namespace rtb;

extern "C" int rtProbe_readBandwidth(uint64_t bytes, int reps, float* out_gbs) {
    clear_error();
    if (bytes < (1u << 20) || reps <= 0 || !out_gbs) {
        set_error("rtProbe_readBandwidth: need at least 1 MiB, reps > 0 and an output");
        return RT_ERR_INVALID;
    }
    const size_t n16 = bytes / 16;
    DevBuf<uint4> buf;
    DevBuf<uint32_t> sink;
    if (!buf.alloc(n16) || !sink.alloc(1)) return RT_ERR_NOMEM;
    // a zero fill: every XOR is zero, never the sink value
    if (!RT_CUDA(cudaMemset(buf.p, 0, n16 * 16))) return RT_ERR_CUDA;
    int per_sm = 0;
    if (!RT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_probe_read, PROBE_T, 0))) return RT_ERR_CUDA;
    const int grid = std::max(1, per_sm) * num_sms();
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!RT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking))) return RT_ERR_CUDA;
    bool ok = RT_CUDA(cudaEventCreate(&e0)) && RT_CUDA(cudaEventCreate(&e1));
    if (ok) {  // warm-up passes (and, for a small buffer, fill L2)
        k_probe_read<<<grid, PROBE_T, 0, s>>>(buf.p, n16, 2, sink.p);
        ok = RT_CUDA(cudaGetLastError());
    }
    ok = ok && RT_CUDA(cudaEventRecord(e0, s));
    if (ok) {
        k_probe_read<<<grid, PROBE_T, 0, s>>>(buf.p, n16, reps, sink.p);
        ok = RT_CUDA(cudaGetLastError());
    }
    ok = ok && RT_CUDA(cudaEventRecord(e1, s)) && RT_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    if (ok) ok = RT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (!ok) return RT_ERR_CUDA;
    *out_gbs = ms > 0.f ? (float)((double)n16 * 16.0 * reps / (ms * 1e-3) / 1e9) : 0.f;
    return RT_OK;
}
