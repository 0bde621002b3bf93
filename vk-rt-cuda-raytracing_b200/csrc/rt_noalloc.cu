// rt_noalloc.cu -- closest-hit trace of a host ray batch that allocates no
// memory: cudaBVH_traceClosestHostNoAlloc.
//
// Who needs it: callers that must not allocate device memory while they
// trace.  A Vulkan layer tracing from inside vkQueueSubmit / present runs on
// the application's render thread, where a cudaMalloc (which may synchronise
// the whole device) would stall the frame, and where the application, not
// the layer, owns the memory budget; real-time or latency-critical callers
// avoid the implicit synchronisation of cudaMalloc/cudaFree; and code that
// runs while another library holds the allocator (or under a strict memory
// cap) cannot grow its own staging buffers.  cudaBVH_traceClosestHost grows
// handle-owned staging buffers on demand; this variant instead stages rays
// and hits in one fixed, file-scope device array.
//
// The scratch array lives in every GPU that loads the library until the
// process exits (kMaxRays x 48 bytes + 256, about 3 MiB).  All calls share
// it: two calls whose GPU work overlaps (different threads or streams)
// overwrite each other's rays and hits, so callers serialise them.  The work
// counter and status word are cleared by every call; the ray and hit areas
// keep the previous call's contents until overwritten.
#include <mutex>

#include "rt_internal.h"
#include "rt_legacy.h"
#include "rt_trace.cuh"

namespace {

constexpr int kMaxRays = 65536;

struct NoAllocScratch {
    RtRay rays[kMaxRays];
    RtHit hits[kMaxRays];
    int work;    // ray counter of the persistent kernel, cleared per call
    int status;  // traversal status word, cleared per call
};

static __device__ __align__(256) unsigned char g_scratch[sizeof(NoAllocScratch)];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
NoAllocScratch* g_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device.  In host code
// the symbol is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, once per device, with that device current.
NoAllocScratch* scratch_for_current_device() {
    int dev = -1;
    if (!RT_CUDA(cudaGetDevice(&dev))) return nullptr;
    if (dev < 0 || dev >= kMaxDevices) {
        rtb::set_error("cudaBVH_traceClosestHostNoAlloc: device %d out of range", dev);
        return nullptr;
    }
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        if (!RT_CUDA(cudaGetSymbolAddress(&p, g_scratch))) return nullptr;
        g_addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    return g_addr[dev];
}

}  // namespace

namespace rtb {

void noalloc_forget_current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return;
    }
    std::lock_guard<std::mutex> g(g_mu);
    g_addr[dev] = nullptr;
}

}  // namespace rtb

extern "C" int cudaBVH_traceClosestHostNoAlloc(CudaBVH_t bvh, const RtRay* h_rays, int n, RtHit* h_hits,
                                               void* stream) {
    if (!bvh || n < 0 || (n > 0 && (!h_rays || !h_hits))) {
        rtb::set_error("cudaBVH_traceClosestHostNoAlloc: invalid argument");
        return RT_ERR_INVALID;
    }
    if (n > kMaxRays) {
        rtb::set_error("cudaBVH_traceClosestHostNoAlloc: %d rays exceed the fixed scratch of %d rays; "
                       "split the batch or use cudaBVH_traceClosestHost", n, kMaxRays);
        return RT_ERR_CAPACITY;
    }
    if (n == 0) return RT_OK;
    NoAllocScratch* sc = scratch_for_current_device();
    if (!sc) return RT_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    if (!RT_CUDA(cudaMemcpyAsync(sc->rays, h_rays, sizeof(RtRay) * (size_t)n, cudaMemcpyHostToDevice, s)) ||
        !RT_CUDA(cudaMemsetAsync(&sc->work, 0, 2 * sizeof(int), s)))
        return RT_ERR_CUDA;
    if (rtb::launch_trace_blas(bvh->bvh8, sc->rays, n, sc->hits, nullptr, nullptr, &sc->work, &sc->status, s) !=
        RT_OK)
        return RT_ERR_CUDA;
    int status = 0;
    if (!RT_CUDA(cudaMemcpyAsync(h_hits, sc->hits, sizeof(RtHit) * (size_t)n, cudaMemcpyDeviceToHost, s)) ||
        !RT_CUDA(cudaMemcpyAsync(&status, &sc->status, sizeof(int), cudaMemcpyDeviceToHost, s)) ||
        !RT_CUDA(cudaStreamSynchronize(s)))
        return RT_ERR_CUDA;
    if (status & rtb::RT_STATUS_STACK) {
        rtb::set_error("cudaBVH_traceClosestHostNoAlloc: traversal stack overflow");
        return RT_ERR_STACK;
    }
    return RT_OK;
}
