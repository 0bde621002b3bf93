// rt_internal.h -- host-side structures shared by the library's translation
// units (handles, device buffers, error reporting, launch helpers).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <utility>
#include <string>
#include <vector>

#include "../../include/cuda_bvh_backend.h"
#include "../../include/rt_b200.h"
#include "rt_common.cuh"

namespace rtb {

// ---- error reporting (thread-local last error; no entry point aborts) ----
void set_error(const char* fmt, ...);
void clear_error();
bool cuda_ok(cudaError_t e, const char* what);
#define RT_CUDA(call) ::rtb::cuda_ok((call), #call)

int num_sms();

// Host-side allocation-failure injection for tests (rtDebug_failAllocations):
// true when the allocation about to be made must fail.
bool alloc_fail_injected();

// Device pointers handed to the kernels are read and written with 16-byte
// (rays, hit records), 8-byte or 4-byte vector accesses; a misaligned one
// would fault on the GPU, so entry points reject it first.
inline bool misaligned(const void* p, size_t a) { return p && (reinterpret_cast<uintptr_t>(p) & (a - 1)) != 0; }
bool check_aligned(const char* who, const void* rays, const void* out, size_t out_align);

// ---- a typed device buffer ----
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t pool_stream = nullptr;  // set when the memory came from scratch_pool()
    bool pooled = false;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    bool alloc(size_t count) {
        release();
        if (count == 0) return true;
        if (alloc_fail_injected()) {
            set_error("cudaMalloc of %zu bytes failed (injected)", count * sizeof(T));
            return false;
        }
        if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            set_error("cudaMalloc of %zu bytes failed", count * sizeof(T));
            return false;
        }
        n = count;
        return true;
    }
    // From the scratch pool, ordered on `st` (allocation and release): for
    // buffers that die before the stream's work is done with them.
    bool alloc_on(size_t count, cudaStream_t st);
    bool ensure(size_t count) { return count <= n ? true : alloc(count); }
    void release() {
        if (p) {
            if (pooled) cudaFreeAsync(p, pool_stream);
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
        pooled = false;
    }
    size_t bytes() const { return n * sizeof(T); }
    void swap(DevBuf& o) {
        std::swap(p, o.p);
        std::swap(n, o.n);
        std::swap(pool_stream, o.pool_stream);
        std::swap(pooled, o.pooled);
    }
};

// ---- builder temporaries: stream-ordered, from a pool that keeps memory ----
// The builders need a few bytes to a few GB of scratch per build.  Taking it
// with cudaMalloc/cudaFree maps and unmaps pages on every build, and every
// cudaFree waits for the whole device, so the build's timeline fills with
// idle gaps.  Scratch comes instead from one pool per device that keeps up to
// `RTB200_POOL_KEEP_MB` (default 32768) MB of freed memory for the next
// build; allocation and release are ordered on the build's stream.
cudaMemPool_t scratch_pool();

template <class T>
struct TmpBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    TmpBuf() = default;
    TmpBuf(const TmpBuf&) = delete;
    TmpBuf& operator=(const TmpBuf&) = delete;
    ~TmpBuf() { release(); }
    bool alloc(size_t count, cudaStream_t st) {
        release();
        if (count == 0) return true;
        if (alloc_fail_injected()) {
            set_error("scratch allocation of %zu bytes failed (injected)", count * sizeof(T));
            return false;
        }
        cudaMemPool_t pool = scratch_pool();
        if (!pool || cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), count * sizeof(T), pool, st) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            set_error("scratch allocation of %zu bytes failed", count * sizeof(T));
            return false;
        }
        s = st;
        n = count;
        return true;
    }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

template <class T>
bool DevBuf<T>::alloc_on(size_t count, cudaStream_t st) {
    release();
    if (count == 0) return true;
    if (alloc_fail_injected()) {
        set_error("scratch allocation of %zu bytes failed (injected)", count * sizeof(T));
        return false;
    }
    cudaMemPool_t pool = scratch_pool();
    if (!pool || cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), count * sizeof(T), pool, st) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        set_error("scratch allocation of %zu bytes failed", count * sizeof(T));
        return false;
    }
    pooled = true;
    pool_stream = st;
    n = count;
    return true;
}

// ---- build configuration ----
struct BuildConfig {
    int max_leaf = 2;        // triangles per BVH2 leaf (1..kMaxLeafTris); the 8-wide
                             // collapse may merge small subtrees into leaves of up to 4
    int small_task = 1024;   // tasks at or below this size finish in one CTA
    int max_sah_depth = 48;  // deeper tasks fall back to median splits
    int warp_task = 32;      // subtrees of at most this many primitives (<= 32) are
                             // finished by one warp with an exact SAH sweep; 0 = off
    bool transient = false;  // the binary tree comes from the scratch pool (a caller
                             // that drops it right after the collapse)
};

// Result of the SAH builder on the device.
struct Bvh2Device {
    DevBuf<Node2> nodes;     // capacity 2N (reserved slots may stay unused)
    DevBuf<int> perm;        // leaf order -> primitive index
    int num_nodes = 0;       // slots used (incl. unused reservations)
    int num_prims = 0;
    int num_roots = 1;       // one root per segment, nodes 0 .. num_roots-1
    void swap(Bvh2Device& o) {
        nodes.swap(o.nodes);
        perm.swap(o.perm);
        std::swap(num_nodes, o.num_nodes);
        std::swap(num_prims, o.num_prims);
        std::swap(num_roots, o.num_roots);
    }
};

// The compressed 8-wide structure the traversal kernels read.
struct Bvh8Device {
    DevBuf<Bvh8Node> nodes;
    DevBuf<TriRec> tris;     // BLAS: triangle records in node order
    DevBuf<int> leaf_ids;    // TLAS: instance index per leaf slot
    int num_nodes = 0;
    int num_leaf_items = 0;
    int depth = 0;
    void swap(Bvh8Device& o) {
        nodes.swap(o.nodes);
        tris.swap(o.tris);
        leaf_ids.swap(o.leaf_ids);
        std::swap(num_nodes, o.num_nodes);
        std::swap(num_leaf_items, o.num_leaf_items);
        std::swap(depth, o.depth);
    }
};

// Defaults with the environment's overrides (RTB200_MAX_LEAF, RTB200_WARP_TASK,
// RTB200_SMALL_TASK).
BuildConfig default_build_config();

// Builds the binary SAH BVH over primitive boxes (lo/hi float4 per prim).
// Returns false on failure (error set).  Stream-ordered; synchronises on
// small counts between levels.
// `segments` (optional, host) splits the primitives into independent scenes
// [seg[i], seg[i+1]) built together; scene i's root is node i.
bool build_bvh2(const float4* d_lo, const float4* d_hi, int n, const BuildConfig& cfg, Bvh2Device& out,
                cudaStream_t s, const std::vector<int>* segments = nullptr);

// Collapses a BVH2 into the 8-wide layout.  For a BLAS d_tris9 holds the
// triangles (9 floats each) and TriRec records are written; for a TLAS
// d_tris9 is null and leaf_ids receives primitive (instance) indices.
bool collapse_bvh8(const Bvh2Device& b2, const float* d_tris9, Bvh8Device& out, cudaStream_t s);

// The whole BLAS build (SAH levels, small and warp tiers, 8-wide collapse)
// as one CUDA graph launched on s: both level loops are conditional WHILE
// nodes driven by counts that stay on the device, so the host neither
// waits between levels nor sizes any launch from a device count.  Same
// tree as build_bvh2 + collapse_bvh8 (segments: scenes built together;
// scene i's root is 8-wide node i).  Returns false with the error set.
struct GraphBuildInfo {
    float graph_ms = 0.f;  // the graph launch, CUDA events on s
    int bvh2_nodes = 0;    // binary node ids used
    int levels = 0;        // large-task levels
    int small_tasks = 0;
};
// Whether the driver runs graphs with conditional nodes (else callers use
// the host-driven loop).
bool graph_build_supported();
// keep (optional): receives the binary tree and permutation (owned buffers)
// for callers that export or refit it; without it they are scratch.
bool build_bvh8_graph(const float4* d_lo, const float4* d_hi, const float* d_tris9, int n, const BuildConfig& cfg,
                      const std::vector<int>& segments, Bvh8Device& out, cudaStream_t s, GraphBuildInfo* info,
                      Bvh2Device* keep = nullptr);
// The same build in two halves, so a caller can capture and launch the next
// build while this one runs: launch_bvh8_graph allocates, captures,
// instantiates and launches on s without waiting (its scratch is released in
// stream order after the graph); finish_bvh8_graph waits for s, reads the
// device counts into `out` (and keep) and checks the build's status.
struct GraphBuildJob {
    TmpBuf<int> result;  // the device counts finish_bvh8_graph reads
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;  // around the graph launch
    cudaGraphExec_t exec = nullptr;
    int n = 0, S = 0;
    Bvh8Device* out = nullptr;
    Bvh2Device* keep = nullptr;
    bool launched = false;
    GraphBuildJob() = default;
    GraphBuildJob(const GraphBuildJob&) = delete;
    GraphBuildJob& operator=(const GraphBuildJob&) = delete;
    ~GraphBuildJob() {
        // an executable graph destroyed while in flight is freed when it completes
        if (exec) cudaGraphExecDestroy(exec);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
};
// d_seg (optional): the segment table already on the device, as absolute
// offsets less seg_base (so nothing is copied from pageable host memory,
// which could wait for the work queued on s).
bool launch_bvh8_graph(const float4* d_lo, const float4* d_hi, const float* d_tris9, int n, const BuildConfig& cfg,
                       const std::vector<int>& segments, Bvh8Device& out, cudaStream_t s, GraphBuildJob& job,
                       Bvh2Device* keep = nullptr, const int* d_seg = nullptr, int seg_base = 0);
bool finish_bvh8_graph(GraphBuildJob& job, GraphBuildInfo* info);

// Capture helpers for the graph-driven build: a conditional handle on the
// graph being captured on cs, and a WHILE node on it at the capture
// position (its empty body graph returned for capture on another stream).
bool capture_conditional_handle(cudaStream_t cs, cudaGraphConditionalHandle* h);
bool capture_while(cudaStream_t cs, cudaGraphConditionalHandle h, cudaGraph_t* body);

// Exclusive scan whose element count is read on the device (d_n; null: all
// `cap` elements), with caller scratch of scan_scratch_ints(cap) ints; no
// allocation, so it can be captured.
size_t scan_scratch_ints(int cap);
bool scan_exclusive_dev(const int* d_in, int* d_out, int cap, const int* d_n, int* d_total, int* scratch,
                        cudaStream_t s);

// The collapse enqueued on a capturing stream cs (its level loop a WHILE
// node whose body is captured on bs), over a binary tree of at most `slots`
// node ids (unused ids zeroed) with R roots; scratch of at least
// collapse_graph_scratch_bytes; d_result receives {nodes, leaf items,
// depth, status (1: capacity exceeded)}.
size_t collapse_graph_scratch_bytes(int n, int R, int slots, bool dp);
bool enqueue_collapse_graph(const Node2* nodes2, const int* perm, int n, int R, int slots, const float* d_tris9,
                            Bvh8Node* out_nodes, TriRec* out_tris, int* out_ids, char* scratch, size_t scratch_bytes,
                            int* d_result, cudaStream_t cs, cudaStream_t bs);

// Primitive boxes.
void launch_tri_bounds(const float* d_tris9, int n, float4* d_lo, float4* d_hi, cudaStream_t s);

// Exclusive scan of n ints (device), total written to *d_total if non-null.
bool scan_exclusive(const int* d_in, int* d_out, int n, int* d_total, cudaStream_t s);

// Host structural check of an 8-wide structure with roots 0 .. num_roots-1
// (error set on failure).
bool validate_bvh8(const Bvh8Device& b, int num_items, int num_prims, int num_roots = 1);

// SAH cost (root-area normalised) of a BVH2.
float bvh2_sah_cost(const Bvh2Device& b2, cudaStream_t s);

}  // namespace rtb

namespace rtb {
// Copy-in / trace / copy-out pipeline of the host-buffer entry points:
// non-blocking streams for copy-in, trace (two, alternating) and copy-out,
// and an event per piece and stage.
struct HostPipe {
    static constexpr int kMaxPieces = 16;
    cudaStream_t in = nullptr, comp[2] = {nullptr, nullptr}, out = nullptr;
    cudaEvent_t start = nullptr, ev_in[kMaxPieces] = {}, ev_tr[kMaxPieces] = {};
    bool ready = false;
    bool init();
    ~HostPipe();
};
}  // namespace rtb

// ---- the handle behind CudaBVH_t ----
struct CudaBVHHandle {
    int num_tris = 0;
    int device = 0;               // the CUDA device current when the handle was created
    float bmin[3], bmax[3], center[3], extent = 0.f;
    rtb::DevBuf<float> tris9;     // input triangles (device copy)
    rtb::Bvh2Device bvh2;
    rtb::Bvh8Device bvh8;
    RtBuildStats stats{};
    std::mutex mu;                // guards lazy host exports and staging
    // lazily built host exports for the layer's Vulkan path
    std::vector<uint32_t> h_dfs;
    std::vector<float> h_packed;
    std::vector<unsigned char> h_bvh4;
    std::vector<float> h_soa[9];
    bool exports_ready = false;
    int num_bvh4 = -1;
    // per-call scratch: work counters (ring; the index is taken atomically so
    // host threads tracing one handle draw distinct slots) and host staging
    rtb::DevBuf<int> counters;
    std::atomic<unsigned> counter_next{0};
    rtb::DevBuf<RtRay> stage_rays;
    rtb::DevBuf<RtHit> stage_hits;
    rtb::DevBuf<uint8_t> stage_occ;
    rtb::DevBuf<float> stage_f;
    rtb::DevBuf<int> status;      // device status word (overflow / errors)
    rtb::HostPipe pipe;           // host-buffer entry points
};

struct CudaTLASHandle {
    int num_instances = 0;
    std::vector<CudaBVH_t> blas;
    rtb::Bvh2Device bvh2;
    rtb::Bvh8Device bvh8;
    rtb::DevBuf<float4> inst;     // per instance: inv xform (3 float4), BLAS ptrs, id base
    std::vector<float> h_inv;     // 12 floats per instance
    std::vector<float> h_fwd;     // 12 floats per instance: the object -> world transforms
    std::vector<int> h_blas;      // BLAS index per instance
    std::atomic<unsigned long long> generation{0};  // bumped by every cudaTLAS_setTransforms
    rtb::DevBuf<int> counters;
    std::atomic<unsigned> counter_next{0};
    rtb::DevBuf<int> status;
    // held by cudaTLAS_setTransforms while it swaps the instances and the top
    // level, and by every trace and render while it launches on them
    std::mutex mu;
};

namespace rtb {
// A new handle for n triangles (h->tris9 not yet allocated), and the build of
// a handle whose device triangles h->tris9 are in place (BVH2, 8-wide
// collapse, statistics, per-call scratch); false with the error set.
CudaBVHHandle* create_handle(int n);
bool build_handle(CudaBVHHandle* h, cudaStream_t s);
// Two-level trace; n_dev (optional) supplies the ray count from device memory.
int launch_trace_tlas(const CudaTLASHandle* t, const RtRay* rays, int n, const int* n_dev, RtHit* hits,
                      int32_t* inst_out, uint8_t* occ, int* work, int* status, cudaStream_t s);
int* next_counter(rtb::DevBuf<int>& ring, std::atomic<unsigned>& next, cudaStream_t s);
// Stable radix sort of rays[0 .. n) by regrouping key into out (payload
// gathered alongside, perm[k] = source index; both optional); n from d_n
// when given (at most cap).  Scratch from the stream-ordered pool.
bool regroup_rays(const RtRay* rays, const int* payload, int cap, const int* d_n, int n_host, const float* box6,
                  int kind, int key_bits, RtRay* out, int* payload_out, int32_t* perm, cudaStream_t s);
// Reads and clears a handle's status word once `s` has finished its work:
// RT_OK, RT_ERR_STACK (some trace overflowed its stack) or RT_ERR_CUDA.
int read_status(int* d_status, cudaStream_t s, const char* who);
// Forgets the cached device address of the allocation-free entry point's
// scratch array on the current device (a device reset invalidates it).
void noalloc_forget_current_device();
bool ensure_counters(rtb::DevBuf<int>& ring);
}  // namespace rtb
