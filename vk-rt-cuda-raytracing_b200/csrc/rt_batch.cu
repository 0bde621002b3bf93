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
    int groups = 1;           // scene groups built one after another (the upload overlapped)
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

// ---- scene groups: the build overlapped with the triangles' upload ----
// A batch of at least kGroupMinTris triangles is built as two groups of
// whole scenes, one build after the other on the build stream, while the
// copy stream brings the next group's triangles across PCIe: the first
// group holds about kFirstShare of the triangles, so its upload is short
// and its build hides the upload of the rest.  Measured on 256 scenes /
// 22.1M triangles: the upload takes 14.3 ms and one build over all scenes
// 30.8 ms of kernels, two groups 16.6 + 16.3 ms, three 35.2 ms in all.
// RTB200_BATCH_GROUPS=<g> sets the number of groups (1: one build over all
// scenes); groups above two split what the first leaves evenly.
constexpr int kGroupMinTris = 8 << 20;
constexpr double kFirstShare = 0.3;
constexpr int kMaxGroups = 8;

std::vector<int> scene_groups(const std::vector<int>& tri_off, int num_scenes) {
    const long long n = tri_off[num_scenes];
    int g = (n >= kGroupMinTris && num_scenes >= 2) ? 2 : 1;
    if (const char* e = getenv("RTB200_BATCH_GROUPS")) g = atoi(e);
    g = std::max(1, std::min({g, num_scenes, kMaxGroups}));
    std::vector<int> bounds{0};
    for (int k = 1; k < g; k++) {
        const double share = kFirstShare + (1.0 - kFirstShare) * (double)(k - 1) / (double)(g - 1);
        const long long target = (long long)(share * (double)n);
        int i = bounds.back() + 1;  // at least one scene per group
        while (i < num_scenes - (g - k) && tri_off[i] < target) i++;
        bounds.push_back(i);
    }
    bounds.push_back(num_scenes);
    return bounds;
}

// Group nodes into the batch layout: the group's scene roots (its nodes
// 0 .. S_g-1) go to root_off + j, its other nodes after all roots, to
// inner_off + (j - S_g); child bases move with the inner nodes and triangle
// bases by rec_off.  A node without inner children keeps its child base.
__global__ void k_merge_nodes(const uint4* __restrict__ src, uint4* __restrict__ dst, int count, int s_g,
                              uint32_t root_off, uint32_t inner_off, uint32_t rec_off) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const uint4* a = src + (size_t)j * 5;
    uint4* b = dst + (size_t)(j < s_g ? root_off + (uint32_t)j : inner_off + (uint32_t)(j - s_g)) * 5;
    const uint4 w0 = a[0];
    uint4 w1 = a[1];
    if (w0.w >> 24) w1.x = w1.x - (uint32_t)s_g + inner_off;
    w1.y += rec_off;
    b[0] = w0;
    b[1] = w1;
    b[2] = a[2];
    b[3] = a[3];
    b[4] = a[4];
}

// Group triangle records after the earlier groups' records; primitive ids
// (group-relative) become batch-relative.
__global__ void k_merge_recs(const TriRec* __restrict__ src, TriRec* __restrict__ dst, int count, int prim_off) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    TriRec r = src[j];
    r.a.w = __int_as_float(__float_as_int(r.a.w) + prim_off);
    dst[j] = r;
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
    const std::vector<int> grp = scene_groups(b->tri_off, num_scenes);
    const int G = (int)grp.size() - 1;
    b->graph_build = !(flags & RT_BATCH_BUILD_HOST_LOOP) && graph_build_supported();
    b->groups = G;
    // page-locked input: every group's copy is queued at once; otherwise a
    // group's copy is issued after the previous group's build is launched
    cudaPointerAttributes pa{};
    const cudaError_t pe = cudaPointerGetAttributes(&pa, h_tris);
    if (pe != cudaSuccess) cudaGetLastError();  // clear only this query's own failure
    const bool pinned = pe == cudaSuccess && pa.type == cudaMemoryTypeHost;
    // the input triangles and the binary trees are needed only while building:
    // pooled scratch, gone when the build returns
    TmpBuf<float> tris9;
    TmpBuf<float4> lo, hi;
    std::vector<Bvh8Device> outs(G);
    std::vector<Bvh2Device> bvh2(b->graph_build ? 0 : G);
    std::vector<GraphBuildJob> jobs(G);
    std::vector<GraphBuildInfo> gi(G);
    std::vector<cudaEvent_t> ev(4 * G + 3, nullptr);  // per group: copied, boxes start / end, build end; merge
    cudaStream_t cp = nullptr;
    bool ok = RT_CUDA(cudaStreamCreateWithFlags(&cp, cudaStreamNonBlocking));
    for (size_t i = 0; ok && i < ev.size(); i++) ok = RT_CUDA(cudaEventCreate(&ev[i]));
    cudaEvent_t* ev_in = ev.data();
    cudaEvent_t* ev_b0 = ev.data() + G;
    cudaEvent_t* ev_b1 = ev.data() + 2 * G;
    cudaEvent_t* ev_end = ev.data() + 3 * G;
    cudaEvent_t ev_ready = ev[4 * G], ev_m0 = ev[4 * G + 1], ev_m1 = ev[4 * G + 2];
    ok = ok && tris9.alloc((size_t)n * 9, s) && b->d_tri_off.alloc(num_scenes + 1) && lo.alloc(n, s) &&
         hi.alloc(n, s) && b->work.alloc(2) && b->status.alloc(1) &&
         RT_CUDA(cudaMemcpyAsync(b->d_tri_off.p, tri_offsets, sizeof(int) * (num_scenes + 1),
                                 cudaMemcpyHostToDevice, s)) &&
         RT_CUDA(cudaMemsetAsync(b->status.p, 0, sizeof(int), s)) && RT_CUDA(cudaEventRecord(ev_ready, s)) &&
         RT_CUDA(cudaStreamWaitEvent(cp, ev_ready, 0));
    auto copy_group = [&](int g) {
        const size_t t0 = (size_t)tri_offsets[grp[g]], t1 = (size_t)tri_offsets[grp[g + 1]];
        return RT_CUDA(cudaMemcpyAsync(tris9.p + t0 * 9, h_tris + t0, sizeof(CudaTri) * (t1 - t0),
                                       cudaMemcpyHostToDevice, cp)) &&
               RT_CUDA(cudaEventRecord(ev_in[g], cp));
    };
    for (int g = 0; ok && pinned && g < G; g++) ok = copy_group(g);
    BuildConfig cfg = default_build_config();
    cfg.transient = true;
    for (int g = 0; ok && g < G; g++) {
        const int t0 = tri_offsets[grp[g]], ng = tri_offsets[grp[g + 1]] - t0;
        std::vector<int> seg(grp[g + 1] - grp[g] + 1);
        for (size_t k = 0; k < seg.size(); k++) seg[k] = tri_offsets[grp[g] + (int)k] - t0;
        ok = (pinned || copy_group(g)) && RT_CUDA(cudaStreamWaitEvent(s, ev_in[g], 0)) &&
             RT_CUDA(cudaEventRecord(ev_b0[g], s));
        if (!ok) break;
        launch_tri_bounds(tris9.p + (size_t)t0 * 9, ng, lo.p + t0, hi.p + t0, s);
        ok = RT_CUDA(cudaEventRecord(ev_b1[g], s));
        // a group's output is scratch for the merge: from the pool, which
        // keeps the memory for the next build
        if (ok && G > 1) {
            const int sg = grp[g + 1] - grp[g];
            ok = outs[g].nodes.alloc_on((size_t)ng + sg, s) && outs[g].tris.alloc_on((size_t)ng, s);
        }
        if (ok && b->graph_build)
            ok = launch_bvh8_graph(lo.p + t0, hi.p + t0, tris9.p + (size_t)t0 * 9, ng, cfg, seg, outs[g], s, jobs[g],
                                   nullptr, b->d_tri_off.p + grp[g], t0);
        else if (ok)
            ok = build_bvh2(lo.p + t0, hi.p + t0, ng, cfg, bvh2[g], s, &seg) &&
                 collapse_bvh8(bvh2[g], tris9.p + (size_t)t0 * 9, outs[g], s);
        ok = ok && RT_CUDA(cudaEventRecord(ev_end[g], s));
    }
    for (int g = 0; ok && b->graph_build && g < G; g++) ok = finish_bvh8_graph(jobs[g], &gi[g]);
    if (ok && G == 1) {
        b->bvh8.swap(outs[0]);
    } else if (ok) {
        // one layout: every scene's root first (scene i at node i), then each
        // group's other nodes; records in group order
        long long nodes = 0, recs = 0;
        int depth = 0;
        for (int g = 0; g < G; g++) {
            nodes += outs[g].num_nodes;
            recs += outs[g].num_leaf_items;
            depth = std::max(depth, outs[g].depth);
        }
        ok = nodes < INT32_MAX && recs == n && b->bvh8.nodes.alloc((size_t)nodes) && b->bvh8.tris.alloc((size_t)recs) &&
             RT_CUDA(cudaEventRecord(ev_m0, s));
        uint32_t inner = (uint32_t)num_scenes, rec = 0;
        for (int g = 0; ok && g < G; g++) {
            const int cnt = outs[g].num_nodes, sg = grp[g + 1] - grp[g], nr = outs[g].num_leaf_items;
            k_merge_nodes<<<(cnt + 255) / 256, 256, 0, s>>>(reinterpret_cast<const uint4*>(outs[g].nodes.p),
                                                           reinterpret_cast<uint4*>(b->bvh8.nodes.p), cnt, sg,
                                                           (uint32_t)grp[g], inner, rec);
            k_merge_recs<<<(nr + 255) / 256, 256, 0, s>>>(outs[g].tris.p, b->bvh8.tris.p + rec, nr,
                                                          tri_offsets[grp[g]]);
            ok = RT_CUDA(cudaGetLastError());
            inner += (uint32_t)(cnt - sg);
            rec += (uint32_t)nr;
        }
        ok = ok && RT_CUDA(cudaEventRecord(ev_m1, s));
        b->bvh8.num_nodes = (int)nodes;
        b->bvh8.num_leaf_items = (int)recs;
        b->bvh8.depth = depth;
    }
    // nothing may still read the scratch or the copies when it is released
    if (cp) ok = RT_CUDA(cudaStreamSynchronize(cp)) && ok;
    ok = RT_CUDA(cudaStreamSynchronize(s)) && ok;
    if (ok) {
        // device time of the build kernels: per group the triangle boxes and
        // the graph launch (the host's capture and instantiation excluded) or
        // the host-driven loop's span, plus the merge
        float ms = 0.f, t = 0.f;
        for (int g = 0; g < G; g++) {
            cudaEventElapsedTime(&t, ev_b0[g], ev_b1[g]);
            ms += t;
            if (b->graph_build) {
                ms += gi[g].graph_ms;
            } else {
                cudaEventElapsedTime(&t, ev_b1[g], ev_end[g]);
                ms += t;
            }
        }
        if (G > 1) {
            cudaEventElapsedTime(&t, ev_m0, ev_m1);
            ms += t;
        }
        b->build_ms = ms;
    }
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    if (cp) cudaStreamDestroy(cp);
    if (ok && getenv("RTB200_VALIDATE") && atoi(getenv("RTB200_VALIDATE")))
        ok = validate_bvh8(b->bvh8, b->bvh8.num_leaf_items, n, num_scenes);
    if (!ok) {
        delete b;
        return nullptr;
    }
    return b;
}

int rtDebug_batchGroups(const int* tri_offsets, int num_scenes, int* out_bounds, int max_groups) {
    if (!tri_offsets || !out_bounds || num_scenes <= 0 || max_groups < 1 || tri_offsets[0] != 0) {
        set_error("rtDebug_batchGroups: invalid argument");
        return RT_ERR_INVALID;
    }
    for (int i = 0; i < num_scenes; i++)
        if (tri_offsets[i + 1] <= tri_offsets[i]) {
            set_error("rtDebug_batchGroups: scene %d has no triangles", i);
            return RT_ERR_INVALID;
        }
    const std::vector<int> g = scene_groups(std::vector<int>(tri_offsets, tri_offsets + num_scenes + 1), num_scenes);
    if ((int)g.size() - 1 > max_groups) {
        set_error("rtDebug_batchGroups: %d groups, room for %d", (int)g.size() - 1, max_groups);
        return RT_ERR_INVALID;
    }
    std::copy(g.begin(), g.end(), out_bounds);
    return (int)g.size() - 1;
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
