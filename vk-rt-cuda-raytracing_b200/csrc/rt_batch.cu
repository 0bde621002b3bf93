// rt_batch.cu -- many independent scenes built and traced together (the
// batched form): every scene's root task enters the same level-synchronous
// SAH pipeline (scene i's root is node i), so all builds share each builder
// stage's launches; all ray batches are traced by one persistent,
// work-stealing launch in which every lane starts at its own scene's root;
// that launch can be captured once into a CUDA graph and replayed.  The
// autotuner times the launch shape on the caller's batch (persistent worker
// warps, node visits per iteration, threads per CTA, shared stack entries)
// and keeps the fastest.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rt_internal.h"
#include "rt_legacy.h"
#include "rt_trace.cuh"

using namespace rtb;

struct RtBatchHandle {
    int num_scenes = 0;
    int num_tris = 0;
    std::vector<int> tri_off;
    DevBuf<int> d_tri_off;
    Bvh8Device bvh8;
    DevBuf<int> work, status;  // work[0]: plain launches, work[1]: graph launches
    RtBatchTuning tune{TRACE_MINB * TRACE_T / 32, RTB_NODE_ITERS, TRACE_T, SSTACK};
    float build_ms = 0.f;
    bool graph_build = true;  // built by the graph-driven builder (else the host-driven level loop)
    // captured graph and the arguments it was captured with
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t cap_stream = nullptr;
    const void* g_rays = nullptr;
    const void* g_off = nullptr;
    void* g_out = nullptr;
    int g_n = -1, g_any = -1;
    RtBatchTuning g_tune{-1, -1, -1, -1};
    ~RtBatchHandle() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (cap_stream) cudaStreamDestroy(cap_stream);
    }
};

namespace {

bool valid_tuning(const RtBatchTuning& t) {
    return t.warps_per_sm >= 1 && t.warps_per_sm <= 64 && t.node_iters >= 1 && t.node_iters <= 4 &&
           (t.block == 64 || t.block == 128 || t.block == 256) &&
           (t.shared_stack == 4 || t.shared_stack == 8 || t.shared_stack == 12);
}

bool tune_from_cache(RtBatchHandle* b, int n) {
    const char* path = getenv("RTB200_TUNE_CACHE");
    if (!path) return false;
    FILE* f = fopen(path, "r");
    if (!f) return false;
    char key[128];
    snprintf(key, sizeof(key), "\"batch:%d:%d:%d\"", b->num_scenes, b->num_tris, n);
    char line[512];
    bool found = false;
    while (fgets(line, sizeof(line), f)) {
        const char* k = strstr(line, key);
        if (!k) continue;
        RtBatchTuning t;
        if (sscanf(k + strlen(key), " : [%d, %d, %d, %d]", &t.warps_per_sm, &t.node_iters, &t.block,
                   &t.shared_stack) == 4 &&
            valid_tuning(t)) {
            b->tune = t;
            found = true;
        }
    }
    fclose(f);
    return found;
}

void tune_to_cache(const RtBatchHandle* b, int n) {
    const char* path = getenv("RTB200_TUNE_CACHE");
    if (!path) return;
    FILE* f = fopen(path, "a");
    if (!f) return;
    fprintf(f, "{\"batch:%d:%d:%d\" : [%d, %d, %d, %d]}\n", b->num_scenes, b->num_tris, n, b->tune.warps_per_sm,
            b->tune.node_iters, b->tune.block, b->tune.shared_stack);
    fclose(f);
}

int check_trace_args(RtBatchHandle* b, const RtRay* rays, const int* off, int n, const void* out, const char* who) {
    if (!b || n < 0 || (n > 0 && (!rays || !off || !out))) {
        set_error("%s: invalid argument", who);
        return RT_ERR_INVALID;
    }
    // closest-hit results are 16-byte records; any-hit results are bytes
    if (!check_aligned(who, rays, off, 4) || misaligned(out, 16)) {
        set_error("%s: device rays and results must be 16-byte aligned, offsets 4-byte aligned", who);
        return RT_ERR_INVALID;
    }
    return RT_OK;
}

}  // namespace

extern "C" {

RtBatch_t rtBatch_buildEx(const CudaTri* h_tris, const int* tri_offsets, int num_scenes, int flags, void* stream) {
    clear_error();
    if (!h_tris || !tri_offsets || num_scenes <= 0 || tri_offsets[0] != 0 ||
        (flags & ~(RT_BATCH_BUILD_HOST_LOOP)) != 0) {
        set_error("rtBatch_build: invalid argument");
        return nullptr;
    }
    for (int i = 0; i < num_scenes; i++)
        if (tri_offsets[i + 1] <= tri_offsets[i]) {
            set_error("rtBatch_build: scene %d has no triangles", i);
            return nullptr;
        }
    cudaStream_t s = (cudaStream_t)stream;
    RtBatchHandle* b = new (std::nothrow) RtBatchHandle();
    if (!b) return nullptr;
    b->num_scenes = num_scenes;
    b->num_tris = tri_offsets[num_scenes];
    b->tri_off.assign(tri_offsets, tri_offsets + num_scenes + 1);
    const int n = b->num_tris;
    // the input triangles and the binary tree are needed only while building:
    // pooled scratch and a local tree, gone when the build returns
    TmpBuf<float> tris9;
    TmpBuf<float4> lo, hi;
    Bvh2Device bvh2;
    cudaEvent_t e0, eb, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&eb);
    cudaEventCreate(&e1);
    bool ok = tris9.alloc((size_t)n * 9, s) && b->d_tri_off.alloc(num_scenes + 1) && lo.alloc(n, s) && hi.alloc(n, s) &&
              b->work.alloc(2) && b->status.alloc(1) &&
              RT_CUDA(cudaMemcpyAsync(tris9.p, h_tris, sizeof(CudaTri) * (size_t)n, cudaMemcpyHostToDevice, s)) &&
              RT_CUDA(cudaMemcpyAsync(b->d_tri_off.p, tri_offsets, sizeof(int) * (num_scenes + 1),
                                      cudaMemcpyHostToDevice, s)) &&
              RT_CUDA(cudaMemsetAsync(b->status.p, 0, sizeof(int), s));
    if (ok) {
        cudaEventRecord(e0, s);
        launch_tri_bounds(tris9.p, n, lo.p, hi.p, s);
        cudaEventRecord(eb, s);
        BuildConfig cfg = default_build_config();
        cfg.transient = true;
        b->graph_build = !(flags & RT_BATCH_BUILD_HOST_LOOP) && graph_build_supported();
        GraphBuildInfo gi;
        if (b->graph_build)
            ok = build_bvh8_graph(lo.p, hi.p, tris9.p, n, cfg, b->tri_off, b->bvh8, s, &gi);
        else
            ok = build_bvh2(lo.p, hi.p, n, cfg, bvh2, s, &b->tri_off) && collapse_bvh8(bvh2, tris9.p, b->bvh8, s);
        cudaEventRecord(e1, s);
        ok = ok && RT_CUDA(cudaEventSynchronize(e1));
        // device time: triangle boxes + the graph launch (capture and
        // instantiation on the host excluded), or the host loop's span
        if (ok && !b->graph_build) cudaEventElapsedTime(&b->build_ms, e0, e1);
        if (ok && b->graph_build) {
            cudaEventElapsedTime(&b->build_ms, e0, eb);
            b->build_ms += gi.graph_ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(eb);
    cudaEventDestroy(e1);
    if (ok && getenv("RTB200_VALIDATE") && atoi(getenv("RTB200_VALIDATE")))
        ok = validate_bvh8(b->bvh8, b->bvh8.num_leaf_items, n, num_scenes);
    if (!ok) {
        delete b;
        return nullptr;
    }
    return b;
}

RtBatch_t rtBatch_build(const CudaTri* h_tris, const int* tri_offsets, int num_scenes, void* stream) {
    return rtBatch_buildEx(h_tris, tri_offsets, num_scenes, 0, stream);
}

void rtBatch_destroy(RtBatch_t b) {
    if (!b) return;
    cudaDeviceSynchronize();
    delete b;
}

int rtBatch_traceClosest(RtBatch_t b, const RtRay* d_rays, const int* d_ray_offsets, int n, RtHit* d_hits,
                         void* stream) {
    int rc = check_trace_args(b, d_rays, d_ray_offsets, n, d_hits, "rtBatch_traceClosest");
    if (rc != RT_OK || n == 0) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(b->work.p, 0, sizeof(int), s);
    rc = launch_trace_multi(b->bvh8, d_rays, n, d_ray_offsets, b->d_tri_off.p, b->num_scenes, d_hits, nullptr,
                            b->work.p, b->status.p, b->tune, s);
    return rc;
}

int rtBatch_traceAny(RtBatch_t b, const RtRay* d_rays, const int* d_ray_offsets, int n, uint8_t* d_occ,
                     void* stream) {
    int rc = check_trace_args(b, d_rays, d_ray_offsets, n, d_occ, "rtBatch_traceAny");
    if (rc != RT_OK || n == 0) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(b->work.p, 0, sizeof(int), s);
    rc = launch_trace_multi(b->bvh8, d_rays, n, d_ray_offsets, b->d_tri_off.p, b->num_scenes, nullptr, d_occ,
                            b->work.p, b->status.p, b->tune, s);
    return rc;
}

int rtBatch_traceGraph(RtBatch_t b, const RtRay* d_rays, const int* d_ray_offsets, int n, void* d_out, int any,
                       void* stream) {
    int rc = check_trace_args(b, d_rays, d_ray_offsets, n, d_out, "rtBatch_traceGraph");
    if (rc != RT_OK || n == 0) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const bool same = b->gexec && b->g_rays == d_rays && b->g_off == d_ray_offsets && b->g_out == d_out &&
                      b->g_n == n && b->g_any == any && memcmp(&b->g_tune, &b->tune, sizeof(RtBatchTuning)) == 0;
    if (!same) {
        if (b->gexec) {
            cudaGraphExecDestroy(b->gexec);
            b->gexec = nullptr;
        }
        if (!b->cap_stream && !RT_CUDA(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking)))
            return RT_ERR_CUDA;
        cudaGraph_t g = nullptr;
        if (!RT_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal))) return RT_ERR_CUDA;
        cudaMemsetAsync(b->work.p + 1, 0, sizeof(int), b->cap_stream);
        const int lrc = launch_trace_multi(b->bvh8, d_rays, n, d_ray_offsets, b->d_tri_off.p, b->num_scenes,
                                           any ? nullptr : (RtHit*)d_out, any ? (uint8_t*)d_out : nullptr,
                                           b->work.p + 1, b->status.p, b->tune, b->cap_stream);
        const bool ended = RT_CUDA(cudaStreamEndCapture(b->cap_stream, &g));
        if (lrc != RT_OK || !ended) {
            if (g) cudaGraphDestroy(g);
            return RT_ERR_CUDA;
        }
        const bool inst = RT_CUDA(cudaGraphInstantiate(&b->gexec, g, 0));
        cudaGraphDestroy(g);
        if (!inst) return RT_ERR_CUDA;
        b->g_rays = d_rays;
        b->g_off = d_ray_offsets;
        b->g_out = d_out;
        b->g_n = n;
        b->g_any = any;
        b->g_tune = b->tune;
    }
    return RT_CUDA(cudaGraphLaunch(b->gexec, s)) ? RT_OK : RT_ERR_CUDA;
}

int rtBatch_autotune(RtBatch_t b, const RtRay* d_rays, const int* d_ray_offsets, int n, RtHit* d_hits,
                     void* stream, int* out_ctas_per_sm, int* out_node_iters) {
    int rc = check_trace_args(b, d_rays, d_ray_offsets, n, d_hits, "rtBatch_autotune");
    if (rc != RT_OK) return rc;
    if (n > 0 && !tune_from_cache(b, n)) {
        cudaStream_t s = (cudaStream_t)stream;
        cudaEvent_t e0, e1;
        if (!RT_CUDA(cudaEventCreate(&e0)) || !RT_CUDA(cudaEventCreate(&e1))) return RT_ERR_CUDA;
        // median of three timed launches after a warm one
        auto time_shape = [&](const RtBatchTuning& t, float& ms_out) -> int {
            b->tune = t;
            int r = rtBatch_traceClosest(b, d_rays, d_ray_offsets, n, d_hits, stream);
            float ms[3];
            for (int k = 0; k < 3 && r == RT_OK; k++) {
                cudaEventRecord(e0, s);
                r = rtBatch_traceClosest(b, d_rays, d_ray_offsets, n, d_hits, stream);
                cudaEventRecord(e1, s);
                if (r == RT_OK && (!RT_CUDA(cudaEventSynchronize(e1)) || !RT_CUDA(cudaEventElapsedTime(&ms[k], e0, e1))))
                    r = RT_ERR_CUDA;
            }
            if (r == RT_OK) ms_out = std::max(std::min(ms[0], ms[1]), std::min(std::max(ms[0], ms[1]), ms[2]));
            return r;
        };
        RtBatchTuning best = b->tune;
        float best_ms = 1e30f;
        rc = time_shape(best, best_ms);
        const int warps[] = {8, 16, 24, 32}, iters[] = {2, 3, 4}, blocks[] = {64, 128, 256}, stacks[] = {4, 8, 12};
        for (int dim = 0; dim < 4 && rc == RT_OK; dim++) {
            const int* vals = dim == 0 ? warps : dim == 1 ? iters : dim == 2 ? blocks : stacks;
            const int nv = dim == 0 ? 4 : 3;
            for (int i = 0; i < nv && rc == RT_OK; i++) {
                RtBatchTuning t = best;
                int& f = dim == 0 ? t.warps_per_sm : dim == 1 ? t.node_iters : dim == 2 ? t.block : t.shared_stack;
                if (f == vals[i]) continue;
                f = vals[i];
                if (dim == 1 && t.node_iters == 3 && (t.block != 128 || t.shared_stack != 8)) continue;
                float ms = 0.f;
                rc = time_shape(t, ms);
                if (rc == RT_OK && ms < best_ms) {
                    best_ms = ms;
                    best = t;
                }
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        b->tune = best;
        if (rc != RT_OK) return rc;
        tune_to_cache(b, n);
    }
    if (out_ctas_per_sm) *out_ctas_per_sm = std::max(1, b->tune.warps_per_sm * 32 / TRACE_T);
    if (out_node_iters) *out_node_iters = b->tune.node_iters;
    return RT_OK;
}

int rtBatch_setTuning(RtBatch_t b, int ctas_per_sm, int node_iters) {
    if (!b || ctas_per_sm < 1 || ctas_per_sm > TRACE_MINB || node_iters < 1 || node_iters > 4) {
        set_error("rtBatch_setTuning: invalid argument");
        return RT_ERR_INVALID;
    }
    b->tune.warps_per_sm = ctas_per_sm * TRACE_T / 32;
    b->tune.node_iters = node_iters;
    return RT_OK;
}

int rtBatch_setTuningEx(RtBatch_t b, const RtBatchTuning* t) {
    if (!b || !t || !valid_tuning(*t)) {
        set_error("rtBatch_setTuningEx: invalid argument");
        return RT_ERR_INVALID;
    }
    b->tune = *t;
    return RT_OK;
}

int rtBatch_getTuning(RtBatch_t b, RtBatchTuning* out) {
    if (!b || !out) {
        set_error("rtBatch_getTuning: invalid argument");
        return RT_ERR_INVALID;
    }
    *out = b->tune;
    return RT_OK;
}

int rtBatch_getDeviceLayout(RtBatch_t b, const void** d_nodes, int* num_nodes, const void** d_tris, int* num_tris) {
    if (!b) {
        set_error("rtBatch_getDeviceLayout: invalid argument");
        return RT_ERR_INVALID;
    }
    if (d_nodes) *d_nodes = b->bvh8.nodes.p;
    if (num_nodes) *num_nodes = b->bvh8.num_nodes;
    if (d_tris) *d_tris = b->bvh8.tris.p;
    if (num_tris) *num_tris = b->bvh8.num_leaf_items;
    return RT_OK;
}

int rtBatch_getInfo(RtBatch_t b, int* num_scenes, int* num_nodes, float* build_ms) {
    if (!b) {
        set_error("rtBatch_getInfo: invalid argument");
        return RT_ERR_INVALID;
    }
    if (num_scenes) *num_scenes = b->num_scenes;
    if (num_nodes) *num_nodes = b->bvh8.num_nodes;
    if (build_ms) *build_ms = b->build_ms;
    return RT_OK;
}

}  // extern "C"
