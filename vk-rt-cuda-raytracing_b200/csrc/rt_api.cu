// rt_api.cu -- the C-ABI: reference-compatible entry points
// (include/cuda_bvh_backend.h) and the extension (include/rt_b200.h).
//
// Every function validates its arguments, reports failures through its
// return value plus rtGetLastError(), and never aborts.  Device work is
// stream-ordered; the reference's per-call cudaMalloc of ray buffers
// (layer/cuda_bvh_backend.cu:1436-1440) is replaced by staging buffers that
// the handle owns and grows on demand.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <thread>

#include "rt_internal.h"
#include "rt_legacy.h"
#include "rt_trace.cuh"

namespace rtb {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    if (getenv("RTB200_LOG")) fprintf(stderr, "[rtb200] %s\n", buf);
}
void clear_error() { g_err.clear(); }
bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    cudaGetLastError();
    set_error("%s: %s", what, cudaGetErrorString(e));
    return false;
}

// Allocations left before injected failures begin; negative = injection off.
static std::atomic<long long> g_alloc_budget{-1};

bool alloc_fail_injected() {
    long long b = g_alloc_budget.load(std::memory_order_relaxed);
    while (b > 0 && !g_alloc_budget.compare_exchange_weak(b, b - 1, std::memory_order_relaxed)) {
    }
    return b == 0;
}

int num_sms() {
    static const int n = [] {
        int d = 0, v = 0;
        cudaGetDevice(&d);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
        return v > 0 ? v : 1;
    }();
    return n;
}

cudaMemPool_t scratch_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        const char* e = getenv("RTB200_POOL_KEEP_MB");
        // at most what the builds used is ever kept; 32 GB holds the whole
        // peak of a 22M-triangle batch built in two groups (about 8.5 GB),
        // whose re-mapping above an 8 GB limit cost 3-4 ms per build
        uint64_t keep = (uint64_t)(e ? std::max(0, atoi(e)) : 32768) << 20;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[dev] = pool;
    }
    return pools[dev];
}

constexpr unsigned kCounterRing = 1024;

bool ensure_counters(DevBuf<int>& ring) {
    if (ring.p) return true;
    if (!ring.alloc(kCounterRing)) return false;
    return RT_CUDA(cudaMemset(ring.p, 0, ring.bytes()));
}

bool check_aligned(const char* who, const void* rays, const void* out, size_t out_align) {
    if (misaligned(rays, 16) || misaligned(out, out_align)) {
        set_error("%s: device rays must be 16-byte aligned and results %zu-byte aligned", who, out_align);
        return false;
    }
    return true;
}

// A fresh zeroed work counter for one launch.  Slots cycle through a ring,
// so up to kCounterRing launches may be in flight on one handle; the index
// is an atomic, so concurrent callers never share a slot.
int* next_counter(DevBuf<int>& ring, std::atomic<unsigned>& next, cudaStream_t s) {
    int* p = ring.p + (next.fetch_add(1, std::memory_order_relaxed) % kCounterRing);
    cudaMemsetAsync(p, 0, sizeof(int), s);
    return p;
}

int read_status(int* d_status, cudaStream_t s, const char* who) {
    int st = 0;
    if (!RT_CUDA(cudaStreamSynchronize(s)) ||
        !RT_CUDA(cudaMemcpy(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost)))
        return RT_ERR_CUDA;
    if (st & RT_STATUS_STACK) {
        set_error("%s: traversal stack overflow", who);
        return RT_CUDA(cudaMemset(d_status, 0, sizeof(int))) ? RT_ERR_STACK : RT_ERR_CUDA;
    }
    return RT_OK;
}

}  // namespace rtb

using namespace rtb;

namespace {

BuildConfig default_config() { return default_build_config(); }

// Builds the handle from device triangles it already owns (h->tris9).
bool build_into(CudaBVHHandle* h, cudaStream_t s) {
    const int n = h->num_tris;
    TmpBuf<float4> lo, hi;
    if (!lo.alloc(n, s) || !hi.alloc(n, s)) return false;
    cudaEvent_t e0, eb, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&eb);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    launch_tri_bounds(h->tris9.p, n, lo.p, hi.p, s);
    cudaEventRecord(eb, s);
    const BuildConfig cfg = default_config();
    // one CUDA graph launch with device-side level loops (the host-driven
    // loop's times swing with the host thread's scheduling: 7.7 ms to 45 ms
    // for the same 2M-triangle build); RTB200_BUILD=host keeps that loop
    static const bool host_loop = [] {
        const char* e = getenv("RTB200_BUILD");
        return (e && !strcmp(e, "host")) || !graph_build_supported();
    }();
    GraphBuildInfo gi;
    bool ok = host_loop ? build_bvh2(lo.p, hi.p, n, cfg, h->bvh2, s) && collapse_bvh8(h->bvh2, h->tris9.p, h->bvh8, s)
                        : build_bvh8_graph(lo.p, hi.p, h->tris9.p, n, cfg, std::vector<int>{0, n}, h->bvh8, s, &gi,
                                           &h->bvh2);
    cudaEventRecord(e1, s);
    if (ok) ok = RT_CUDA(cudaEventSynchronize(e1));
    // device time of the build kernels: the triangle boxes and the graph
    // launch (the host's capture and instantiation in between excluded); the
    // host-driven loop's span on the stream
    float ms = 0.f;
    if (ok && host_loop) cudaEventElapsedTime(&ms, e0, e1);
    if (ok && !host_loop) {
        cudaEventElapsedTime(&ms, e0, eb);
        ms += gi.graph_ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(eb);
    cudaEventDestroy(e1);
    if (!ok) return false;
    Node2 root;
    if (!RT_CUDA(cudaMemcpy(&root, h->bvh2.nodes.p, sizeof(Node2), cudaMemcpyDeviceToHost))) return false;
    for (int a = 0; a < 3; a++) {
        h->bmin[a] = root.lo[a];
        h->bmax[a] = root.hi[a];
        h->center[a] = (root.lo[a] + root.hi[a]) * 0.5f;
    }
    const float ex = h->bmax[0] - h->bmin[0], ey = h->bmax[1] - h->bmin[1], ez = h->bmax[2] - h->bmin[2];
    h->extent = sqrtf(ex * ex + ey * ey + ez * ez);
    RtBuildStats& st = h->stats;
    st.num_tris = n;
    st.num_bvh2_nodes = h->bvh2.num_nodes;
    st.num_nodes = h->bvh8.num_nodes;
    st.depth = h->bvh8.depth;
    st.max_leaf = cfg.max_leaf;
    st.bins = kBins;
    st.build_ms = ms;
    st.sah_cost = bvh2_sah_cost(h->bvh2, s);
    st.node_bytes = (uint64_t)h->bvh8.num_nodes * sizeof(Bvh8Node);
    st.tri_bytes = (uint64_t)h->bvh8.num_leaf_items * sizeof(TriRec);
    if (!ensure_counters(h->counters) || !h->status.alloc(1)) return false;
    if (!RT_CUDA(cudaMemset(h->status.p, 0, sizeof(int)))) return false;
    // structural check before any traversal reads the nodes
    if (getenv("RTB200_VALIDATE") && atoi(getenv("RTB200_VALIDATE")) &&
        !validate_bvh8(h->bvh8, h->bvh8.num_leaf_items, h->num_tris))
        return false;
    return true;
}

CudaBVHHandle* new_handle(int n) {
    CudaBVHHandle* h = new (std::nothrow) CudaBVHHandle();
    if (!h) {
        set_error("out of host memory");
        return nullptr;
    }
    h->num_tris = n;
    if (cudaGetDevice(&h->device) != cudaSuccess) {
        cudaGetLastError();
        h->device = 0;
    }
    return h;
}

// ---- host exports for the layer's Vulkan path (built on first use) ----
uint16_t half_bits(_Float16 x) {
    uint16_t u;
    memcpy(&u, &x, 2);
    return u;
}
float half_val(uint16_t u) {
    _Float16 x;
    memcpy(&x, &u, 2);
    return (float)x;
}
uint16_t half_step(uint16_t u, bool up) {
    // next representable half toward +inf (up) or -inf
    const bool neg = u & 0x8000u;
    if ((u & 0x7FFFu) == 0) return up ? 0x0001u : 0x8001u;
    if (up != neg) return u + 1;
    return u - 1;
}
uint16_t half_down(float x) {  // largest half <= x
    uint16_t h = half_bits((_Float16)x);
    if (half_val(h) > x) h = half_step(h, false);
    return h;
}
uint16_t half_up(float x) {  // smallest half >= x
    uint16_t h = half_bits((_Float16)x);
    if (half_val(h) < x) h = half_step(h, true);
    return h;
}

struct B4 {
    uint16_t bx[8], by[8], bz[8];
    int child[4];
};
static_assert(sizeof(B4) == 64, "BVH4 export node is 64 bytes");

// BVH4 export with the grandchild pull-up of layer/cuda_bvh_backend.cu:391-418
// (preorder numbering, leaf encoding -(start<<3 | count-1) - 2), bounds
// rounded outward to fp16.
int collapse4(const std::vector<Node2>& nd, int ni, std::vector<B4>& out) {
    const Node2& n = nd[ni];
    if (n.b < 0) return -((n.a << 3) | (-n.b - 1)) - 2;
    int gather[4], ng = 0;
    const int ch[2] = {n.a, n.b};
    for (int c = 0; c < 2; c++) {
        const Node2& cn = nd[ch[c]];
        if (cn.b < 0 || ng >= 3) {
            gather[ng++] = ch[c];
            continue;
        }
        gather[ng++] = cn.a;
        gather[ng++] = cn.b;
    }
    B4 b;
    for (int i = 0; i < 4; i++) {
        if (i < ng) {
            const Node2& c = nd[gather[i]];
            b.bx[i] = half_down(c.lo[0]); b.bx[4 + i] = half_up(c.hi[0]);
            b.by[i] = half_down(c.lo[1]); b.by[4 + i] = half_up(c.hi[1]);
            b.bz[i] = half_down(c.lo[2]); b.bz[4 + i] = half_up(c.hi[2]);
        } else {
            b.bx[i] = b.by[i] = b.bz[i] = 0x7C00u;              // +inf
            b.bx[4 + i] = b.by[4 + i] = b.bz[4 + i] = 0xFC00u;  // -inf
        }
        b.child[i] = -1;
    }
    const int me = (int)out.size();
    out.push_back(b);
    for (int i = 0; i < ng; i++) {
        const int c = collapse4(nd, gather[i], out);
        out[me].child[i] = c;
    }
    return me;
}

bool ensure_exports(CudaBVHHandle* h) {
    std::lock_guard<std::mutex> g(h->mu);
    if (h->exports_ready) return true;
    const int n = h->num_tris;
    std::vector<Node2> nd(h->bvh2.num_nodes);
    std::vector<int> perm(n);
    std::vector<float> tris((size_t)n * 9);
    if (!RT_CUDA(cudaMemcpy(nd.data(), h->bvh2.nodes.p, nd.size() * sizeof(Node2), cudaMemcpyDeviceToHost)) ||
        !RT_CUDA(cudaMemcpy(perm.data(), h->bvh2.perm.p, perm.size() * sizeof(int), cudaMemcpyDeviceToHost)) ||
        !RT_CUDA(cudaMemcpy(tris.data(), h->tris9.p, tris.size() * sizeof(float), cudaMemcpyDeviceToHost)))
        return false;
    // preorder + subtree sizes -> stackless export with correct skips
    std::vector<int> order;
    order.reserve(nd.size());
    std::vector<int> st{0};
    while (!st.empty()) {
        const int i = st.back();
        st.pop_back();
        order.push_back(i);
        if (nd[i].b > 0) {
            st.push_back(nd[i].b);
            st.push_back(nd[i].a);
        }
    }
    const int m = (int)order.size();
    std::vector<int> pos(nd.size(), -1), size(nd.size(), 1);
    for (int k = 0; k < m; k++) pos[order[k]] = k;
    for (int k = m - 1; k >= 0; k--) {
        const Node2& x = nd[order[k]];
        if (x.b > 0) size[order[k]] = 1 + size[x.a] + size[x.b];
    }
    h->h_dfs.assign((size_t)m * 8, 0u);
    for (int k = 0; k < m; k++) {
        const Node2& x = nd[order[k]];
        uint32_t* p = &h->h_dfs[(size_t)k * 8];
        memcpy(p, x.lo, 12);
        memcpy(p + 3, x.hi, 12);
        const int enc = x.b < 0 ? -((x.a << 3) | (-x.b - 1)) - 2 : 0;
        const int skip = k + size[order[k]] < m ? k + size[order[k]] : -1;
        memcpy(p + 6, &enc, 4);
        memcpy(p + 7, &skip, 4);
    }
    h->h_packed.assign((size_t)n * 12, 0.f);
    for (int c = 0; c < 9; c++) h->h_soa[c].resize(n);
    for (int i = 0; i < n; i++) {
        const float* t = &tris[(size_t)perm[i] * 9];
        float* p = &h->h_packed[(size_t)i * 12];
        for (int c = 0; c < 9; c++) {
            p[c] = t[c];
            h->h_soa[c][i] = t[c];
        }
        p[9] = (float)perm[i];
    }
    std::vector<B4> b4;
    b4.reserve(nd.size() / 2 + 1);
    collapse4(nd, 0, b4);
    h->h_bvh4.resize(b4.size() * sizeof(B4));
    memcpy(h->h_bvh4.data(), b4.data(), h->h_bvh4.size());
    h->num_bvh4 = (int)b4.size();
    h->exports_ready = true;
    return true;
}

// ---- look-at camera basis of layer/cuda_bvh_backend.cu:994-1016 ----
CamBasis lookat_basis(const CudaBVHHandle* h, float cx, float cy, float cz) {
    CamBasis c;
    c.eye[0] = cx; c.eye[1] = cy; c.eye[2] = cz;
    float fx = h->center[0] - cx, fy = h->center[1] - cy, fz = h->center[2] - cz;
    float fl = sqrtf(fx * fx + fy * fy + fz * fz);
    if (fl < 1e-6f) fl = 1.f;
    fx /= fl; fy /= fl; fz /= fl;
    float rx = fz, ry = 0.f, rz = -fx;
    const float rl = sqrtf(rx * rx + rz * rz);
    if (rl > 1e-6f) { rx /= rl; rz /= rl; } else { rx = 1.f; rz = 0.f; }
    c.fwd[0] = fx; c.fwd[1] = fy; c.fwd[2] = fz;
    c.right[0] = rx; c.right[1] = ry; c.right[2] = rz;
    c.up[0] = ry * fz - rz * fy;
    c.up[1] = rz * fx - rx * fz;
    c.up[2] = rx * fy - ry * fx;
    c.fov = 0.6f;
    return c;
}

// Renders the shaded look-at image into device memory `out` (fmt as in the header).
bool render_rgba(CudaBVHHandle* h, int w, int ht, float cx, float cy, float cz, void* out, int fmt, cudaStream_t s) {
    const int n = w * ht;
    if (!h->stage_rays.ensure(n) || !h->stage_hits.ensure(n)) return false;
    launch_gen_lookat(h->stage_rays.p, w, ht, lookat_basis(h, cx, cy, cz), s);
    int* work = next_counter(h->counters, h->counter_next, s);
    if (launch_trace_blas(h->bvh8, h->stage_rays.p, n, h->stage_hits.p, nullptr, nullptr, work, h->status.p, s) != RT_OK)
        return false;
    launch_shade(h->stage_rays.p, h->stage_hits.p, h->tris9.p, w, ht, out, fmt, s);
    return RT_CUDA(cudaGetLastError());
}

int bytes_per_pixel(int fmt) { return fmt == 3 ? 16 : (fmt == 2 ? 8 : 4); }

// ---- background tracer for traceToHostPtr / traceToGPUAsync ----
struct AsyncTracer {
    std::mutex m;
    std::condition_variable cv_req, cv_done;
    std::thread th;
    bool started = false, running = false, has_req = false, has_result = false;
    CudaBVH_t bvh = nullptr;
    int w = 0, ht = 0, fmt = 0;
    float cx = 0, cy = 0, cz = 0;
    void* gpu_target = nullptr;
    std::vector<unsigned char> host[2];
    int read_idx = 0, write_idx = 1;
    uint64_t size = 0;
    ~AsyncTracer() {
        {
            std::lock_guard<std::mutex> g(m);
            running = false;
        }
        cv_req.notify_all();
        if (th.joinable()) th.join();
    }
    void loop() {
        void* dbuf = nullptr;
        size_t dsize = 0;
        for (;;) {
            std::unique_lock<std::mutex> lk(m);
            cv_req.wait(lk, [&] { return has_req || !running; });
            if (!running) break;
            CudaBVH_t b = bvh;
            const int W = w, H = ht, F = fmt;
            const float X = cx, Y = cy, Z = cz;
            void* tgt = gpu_target;
            const int wi = write_idx;
            const uint64_t sz = size;
            has_req = false;
            lk.unlock();
            bool ok = true;
            if (tgt) {
                ok = render_rgba(b, W, H, X, Y, Z, tgt, F, 0) && RT_CUDA(cudaStreamSynchronize(0));
            } else {
                const size_t need = (size_t)W * H * bytes_per_pixel(F);
                if (dsize < need) {
                    if (dbuf) cudaFree(dbuf);
                    dbuf = nullptr;
                    dsize = 0;
                    if (cudaMalloc(&dbuf, need) == cudaSuccess) dsize = need;
                }
                ok = dbuf && render_rgba(b, W, H, X, Y, Z, dbuf, F, 0) &&
                     RT_CUDA(cudaMemcpy(host[wi].data(), dbuf, std::min<uint64_t>(sz, need), cudaMemcpyDeviceToHost));
            }
            lk.lock();
            if (ok) {
                read_idx = wi;
                write_idx = 1 - wi;
            }
            has_result = true;
            lk.unlock();
            cv_done.notify_all();
        }
        if (dbuf) cudaFree(dbuf);
    }
    void submit(CudaBVH_t b, int W, int H, float X, float Y, float Z, int F, void* tgt, uint64_t sz) {
        std::unique_lock<std::mutex> lk(m);
        if (!started) {
            started = running = true;
            th = std::thread([this] { loop(); });
        }
        if (!tgt && sz != size) {
            host[0].assign(sz, 0);
            host[1].assign(sz, 0);
            size = sz;
        }
        bvh = b; w = W; ht = H; cx = X; cy = Y; cz = Z; fmt = F; gpu_target = tgt;
        has_req = true;
        lk.unlock();
        cv_req.notify_one();
    }
    void wait_first() {
        std::unique_lock<std::mutex> lk(m);
        cv_done.wait(lk, [&] { return has_result; });
    }
};
AsyncTracer g_async;

}  // namespace

namespace rtb {
bool build_handle(CudaBVHHandle* h, cudaStream_t s) { return build_into(h, s); }
CudaBVHHandle* create_handle(int n) { return new_handle(n); }
}  // namespace rtb

namespace rtb {
// Host check of an 8-wide structure: every child index, triangle range and
// grid exponent in bounds, nodes numbered after their parents (acyclic),
// every leaf item referenced exactly once, depth within the stack bound.
bool validate_bvh8(const Bvh8Device& b, int num_items, int num_prims, int num_roots) {
    std::vector<Bvh8Node> nd(b.num_nodes);
    if (!RT_CUDA(cudaMemcpy(nd.data(), b.nodes.p, nd.size() * sizeof(Bvh8Node), cudaMemcpyDeviceToHost))) return false;
    std::vector<int> items(num_items, -1);
    if (b.tris.p) {
        std::vector<TriRec> tr(num_items);
        if (!RT_CUDA(cudaMemcpy(tr.data(), b.tris.p, tr.size() * sizeof(TriRec), cudaMemcpyDeviceToHost))) return false;
        for (int i = 0; i < num_items; i++) memcpy(&items[i], &tr[i].a.w, 4);
    } else if (!RT_CUDA(cudaMemcpy(items.data(), b.leaf_ids.p, items.size() * sizeof(int), cudaMemcpyDeviceToHost))) {
        return false;
    }
    std::vector<int> seen(num_items, 0), depth(b.num_nodes, 0), prim_seen(num_prims, 0);
    if (b.num_nodes < 1) {
        set_error("validate: no nodes");
        return false;
    }
    for (int r = 0; r < num_roots && r < b.num_nodes; r++) depth[r] = 1;
    for (int i = 0; i < b.num_nodes; i++) {
        if (depth[i] == 0) {
            set_error("validate: node %d unreachable", i);
            return false;
        }
        if (depth[i] > SSTACK_TOTAL) {
            set_error("validate: depth %d exceeds the traversal stack", depth[i]);
            return false;
        }
        const uint4* w = nd[i].w;
        const uint32_t imask = w[0].w >> 24;
        for (int a = 0; a < 3; a++) {
            const uint32_t e = (w[0].w >> (8 * a)) & 0xFFu;
            if (e == 255u) {
                set_error("validate: node %d bad exponent", i);
                return false;
            }
        }
        const uint32_t cb = w[1].x, tb = w[1].y;
        int k = 0;
        for (int s = 0; s < 8; s++) {
            const uint32_t meta = ((s < 4 ? w[1].z : w[1].w) >> ((s & 3) * 8)) & 0xFFu;
            if ((imask >> s) & 1u) {
                const uint32_t c = cb + k++;
                if ((int)c <= i || (int)c >= b.num_nodes) {
                    set_error("validate: node %d child %u out of range", i, c);
                    return false;
                }
                depth[c] = depth[i] + 1;
            } else if (meta) {
                const uint32_t cnt = meta >> 5, off = meta & 31u;
                if (off + cnt > 32u || tb + off + cnt > (uint32_t)num_items) {
                    set_error("validate: node %d leaf range out of bounds", i);
                    return false;
                }
                for (uint32_t j = 0; j < cnt; j++) seen[tb + off + j]++;
            }
        }
    }
    for (int i = 0; i < num_items; i++) {
        if (seen[i] != 1 || items[i] < 0 || items[i] >= num_prims || prim_seen[items[i]]++) {
            set_error("validate: leaf item %d referenced %d times (id %d)", i, seen[i], items[i]);
            return false;
        }
    }
    return true;
}
}  // namespace rtb

// ============================================================ C-ABI =====
extern "C" {

const char* rtGetLastError(void) { return g_err.c_str(); }

int cudaBVH_validate(CudaBVH_t h) {
    if (!h) {
        set_error("cudaBVH_validate: invalid argument");
        return RT_ERR_INVALID;
    }
    if (h->bvh8.num_leaf_items != h->num_tris) {
        set_error("validate: %d triangle records for %d triangles", h->bvh8.num_leaf_items, h->num_tris);
        return RT_ERR_INVALID;
    }
    return validate_bvh8(h->bvh8, h->bvh8.num_leaf_items, h->num_tris) ? RT_OK : RT_ERR_INVALID;
}

CudaBVH_t cudaBVH_build(const CudaTri* tris, int numTris) {
    clear_error();
    if (!tris || numTris <= 0) {
        set_error("cudaBVH_build: empty input");
        return nullptr;
    }
    CudaBVHHandle* h = new_handle(numTris);
    if (!h) return nullptr;
    if (!h->tris9.alloc((size_t)numTris * 9) ||
        !RT_CUDA(cudaMemcpy(h->tris9.p, tris, sizeof(CudaTri) * (size_t)numTris, cudaMemcpyHostToDevice)) ||
        !build_into(h, 0)) {
        delete h;
        return nullptr;
    }
    return h;
}

CudaBVH_t cudaBVH_buildDevice(const CudaTri* d_tris, int numTris, void* stream) {
    clear_error();
    if (!d_tris || numTris <= 0) {
        set_error("cudaBVH_buildDevice: empty input");
        return nullptr;
    }
    cudaStream_t s = (cudaStream_t)stream;
    CudaBVHHandle* h = new_handle(numTris);
    if (!h) return nullptr;
    if (!h->tris9.alloc((size_t)numTris * 9) ||
        !RT_CUDA(cudaMemcpyAsync(h->tris9.p, d_tris, sizeof(CudaTri) * (size_t)numTris, cudaMemcpyDeviceToDevice, s)) ||
        !build_into(h, s)) {
        delete h;
        return nullptr;
    }
    return h;
}

void cudaBVH_destroy(CudaBVH_t bvh) {
    if (!bvh) return;
    cudaDeviceSynchronize();
    delete bvh;
}

int cudaBVH_traceClosest(CudaBVH_t h, const RtRay* d_rays, int n, RtHit* d_hits, void* stream) {
    if (!h || n < 0 || (n > 0 && (!d_rays || !d_hits))) {
        set_error("cudaBVH_traceClosest: invalid argument");
        return RT_ERR_INVALID;
    }
    if (!check_aligned("cudaBVH_traceClosest", d_rays, d_hits, 16)) return RT_ERR_INVALID;
    if (n == 0) return RT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    int* work = next_counter(h->counters, h->counter_next, s);
    const int rc = launch_trace_blas(h->bvh8, d_rays, n, d_hits, nullptr, nullptr, work, h->status.p, s);
    return rc;
}

int cudaBVH_traceAny(CudaBVH_t h, const RtRay* d_rays, int n, uint8_t* d_occ, void* stream) {
    if (!h || n < 0 || (n > 0 && (!d_rays || !d_occ))) {
        set_error("cudaBVH_traceAny: invalid argument");
        return RT_ERR_INVALID;
    }
    if (!check_aligned("cudaBVH_traceAny", d_rays, d_occ, 1)) return RT_ERR_INVALID;
    if (n == 0) return RT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    int* work = next_counter(h->counters, h->counter_next, s);
    const int rc = launch_trace_blas(h->bvh8, d_rays, n, nullptr, d_occ, nullptr, work, h->status.p, s);
    return rc;
}

int cudaBVH_traceCounters(CudaBVH_t h, const RtRay* d_rays, int n, int any, uint32_t* d_counts, void* stream) {
    if (!h || n < 0 || (n > 0 && (!d_rays || !d_counts))) {
        set_error("cudaBVH_traceCounters: invalid argument");
        return RT_ERR_INVALID;
    }
    if (!check_aligned("cudaBVH_traceCounters", d_rays, d_counts, 8)) return RT_ERR_INVALID;
    if (n == 0) return RT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    std::lock_guard<std::mutex> g(h->mu);
    if (!h->stage_hits.ensure(n) || !h->stage_occ.ensure(n)) return RT_ERR_NOMEM;
    int* work = next_counter(h->counters, h->counter_next, s);
    return launch_trace_blas(h->bvh8, d_rays, n, any ? nullptr : h->stage_hits.p, any ? h->stage_occ.p : nullptr,
                             d_counts, work, h->status.p, s);
}

static int check_status(CudaBVHHandle* h) { return read_status(h->status.p, 0, "trace"); }

int rtDebug_failAllocations(int after) {
    g_alloc_budget.store(after < 0 ? -1 : after, std::memory_order_relaxed);
    return RT_OK;
}

int cudaBVH_getStatus(CudaBVH_t h, void* stream) {
    if (!h) {
        set_error("cudaBVH_getStatus: invalid argument");
        return RT_ERR_INVALID;
    }
    return read_status(h->status.p, (cudaStream_t)stream, "cudaBVH_getStatus");
}

namespace rtb {

bool HostPipe::init() {
    if (ready) return true;
    bool ok = RT_CUDA(cudaStreamCreateWithFlags(&in, cudaStreamNonBlocking)) &&
              RT_CUDA(cudaStreamCreateWithFlags(&comp[0], cudaStreamNonBlocking)) &&
              RT_CUDA(cudaStreamCreateWithFlags(&comp[1], cudaStreamNonBlocking)) &&
              RT_CUDA(cudaStreamCreateWithFlags(&out, cudaStreamNonBlocking)) &&
              RT_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
    for (int i = 0; ok && i < kMaxPieces; i++)
        ok = RT_CUDA(cudaEventCreateWithFlags(&ev_in[i], cudaEventDisableTiming)) &&
             RT_CUDA(cudaEventCreateWithFlags(&ev_tr[i], cudaEventDisableTiming));
    ready = ok;
    return ok;
}

HostPipe::~HostPipe() {
    for (cudaStream_t s : {in, comp[0], comp[1], out})
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    if (start) cudaEventDestroy(start);
    for (int i = 0; i < kMaxPieces; i++) {
        if (ev_in[i]) cudaEventDestroy(ev_in[i]);
        if (ev_tr[i]) cudaEventDestroy(ev_tr[i]);
    }
}

}  // namespace rtb

namespace {

// Host-buffer trace: the batch is cut into pieces (at least 512K rays by
// default, at most HostPipe::kMaxPieces of them) whose copy in, trace and
// copy out run on separate streams chained by events, so the copy of piece
// k+1 and the results of piece k-1 cross PCIe while piece k is traced.
// Successive traces alternate between two streams, so a piece's launch can
// fill the SMs while the slowest rays of the previous piece finish.
// Ordered after earlier work on the legacy default stream; returns when the
// results are in host memory.
int trace_host(CudaBVHHandle* h, const RtRay* rays, int n, void* out, bool any) {
    std::lock_guard<std::mutex> g(h->mu);
    HostPipe& p = h->pipe;
    if (!p.init()) return RT_ERR_CUDA;
    if (!h->stage_rays.ensure(n) || (any ? !h->stage_occ.ensure(n) : !h->stage_hits.ensure(n))) return RT_ERR_NOMEM;
    // smallest piece: 512K rays unless RTB200_HOST_PIECE says otherwise (read once)
    static const int kMinPiece = [] {
        const char* e = getenv("RTB200_HOST_PIECE");
        const int v = e ? atoi(e) : 0;
        return v >= 4096 ? v : (1 << 19);
    }();
    int piece = std::max(kMinPiece, (n + HostPipe::kMaxPieces - 1) / HostPipe::kMaxPieces);
    piece = (piece + 31) & ~31;
    const size_t es = any ? 1 : sizeof(RtHit);
    char* dev_out = any ? (char*)h->stage_occ.p : (char*)h->stage_hits.p;
    if (!RT_CUDA(cudaEventRecord(p.start, 0)) || !RT_CUDA(cudaStreamWaitEvent(p.in, p.start, 0)))
        return RT_ERR_CUDA;
    int k = 0;
    for (int b = 0; b < n; b += piece, k++) {
        const int c = std::min(piece, n - b);
        cudaStream_t comp = p.comp[k & 1];
        if (!RT_CUDA(cudaMemcpyAsync(h->stage_rays.p + b, rays + b, sizeof(RtRay) * (size_t)c, cudaMemcpyHostToDevice,
                                     p.in)) ||
            !RT_CUDA(cudaEventRecord(p.ev_in[k], p.in)) || !RT_CUDA(cudaStreamWaitEvent(comp, p.ev_in[k], 0)))
            return RT_ERR_CUDA;
        int* work = next_counter(h->counters, h->counter_next, comp);
        const int rc = launch_trace_blas(h->bvh8, h->stage_rays.p + b, c, any ? nullptr : h->stage_hits.p + b,
                                         any ? h->stage_occ.p + b : nullptr, nullptr, work, h->status.p, comp);
        if (rc != RT_OK) return rc;
        if (!RT_CUDA(cudaEventRecord(p.ev_tr[k], comp)) || !RT_CUDA(cudaStreamWaitEvent(p.out, p.ev_tr[k], 0)) ||
            !RT_CUDA(cudaMemcpyAsync((char*)out + (size_t)b * es, dev_out + (size_t)b * es, (size_t)c * es,
                                     cudaMemcpyDeviceToHost, p.out)))
            return RT_ERR_CUDA;
    }
    if (!RT_CUDA(cudaStreamSynchronize(p.out))) return RT_ERR_CUDA;
    return check_status(h);
}

constexpr int kMaxReplicas = 64;  // handles per multi-replica call

// One host-buffer batch over several replicas (one handle per device): the
// rays split into contiguous blocks, as even as possible in handle order,
// each traced by its handle's host pipeline on its own device from its own
// host thread; returns when every block's results are in host memory.  The
// first failing block's code and message are returned.
int trace_host_multi(const CudaBVH_t* bvhs, int count, const RtRay* rays, int n, void* out, bool any,
                     const char* who) {
    if (!bvhs || count < 1 || count > kMaxReplicas || n < 0 || (n > 0 && (!rays || !out))) {
        set_error("%s: invalid argument", who);
        return RT_ERR_INVALID;
    }
    for (int i = 0; i < count; i++)
        if (!bvhs[i]) {
            set_error("%s: handle %d is null", who, i);
            return RT_ERR_INVALID;
        }
    if (n == 0) return RT_OK;
    const size_t es = any ? 1 : sizeof(RtHit);
    std::vector<int> rc(count, RT_OK);
    std::vector<std::string> msg(count);
    std::vector<std::thread> th;
    th.reserve(count);
    const int q = n / count, r = n % count;
    for (int i = 0; i < count; i++) {
        const int first = i * q + std::min(i, r), cnt = q + (i < r ? 1 : 0);
        if (cnt == 0) continue;
        th.emplace_back([&, i, first, cnt] {
            CudaBVHHandle* h = bvhs[i];
            if (!RT_CUDA(cudaSetDevice(h->device))) {
                rc[i] = RT_ERR_CUDA;
            } else {
                rc[i] = trace_host(h, rays + first, cnt, (char*)out + (size_t)first * es, any);
            }
            if (rc[i] != RT_OK) msg[i] = rtGetLastError();
        });
    }
    for (std::thread& t : th) t.join();
    for (int i = 0; i < count; i++)
        if (rc[i] != RT_OK) {
            set_error("%s: replica %d: %s", who, i, msg[i].c_str());
            return rc[i];
        }
    return RT_OK;
}

}  // namespace

int cudaBVH_traceClosestHostMulti(const CudaBVH_t* bvhs, int count, const RtRay* rays, int n, RtHit* hits) {
    return trace_host_multi(bvhs, count, rays, n, hits, false, "cudaBVH_traceClosestHostMulti");
}

int cudaBVH_traceAnyHostMulti(const CudaBVH_t* bvhs, int count, const RtRay* rays, int n, uint8_t* occ) {
    return trace_host_multi(bvhs, count, rays, n, occ, true, "cudaBVH_traceAnyHostMulti");
}

int cudaBVH_traceClosestHost(CudaBVH_t h, const RtRay* rays, int n, RtHit* hits) {
    if (!h || n < 0 || (n > 0 && (!rays || !hits))) {
        set_error("cudaBVH_traceClosestHost: invalid argument");
        return RT_ERR_INVALID;
    }
    if (n == 0) return RT_OK;
    return trace_host(h, rays, n, hits, false);
}

int cudaBVH_traceAnyHost(CudaBVH_t h, const RtRay* rays, int n, uint8_t* occ) {
    if (!h || n < 0 || (n > 0 && (!rays || !occ))) {
        set_error("cudaBVH_traceAnyHost: invalid argument");
        return RT_ERR_INVALID;
    }
    if (n == 0) return RT_OK;
    return trace_host(h, rays, n, occ, true);
}

int cudaBVH_getBuildStats(CudaBVH_t h, RtBuildStats* out) {
    if (!h || !out) {
        set_error("cudaBVH_getBuildStats: invalid argument");
        return RT_ERR_INVALID;
    }
    *out = h->stats;
    return RT_OK;
}

int cudaBVH_getDeviceLayout(CudaBVH_t h, const void** d_nodes, int* num_nodes, const void** d_tris, int* num_tris) {
    if (!h) {
        set_error("cudaBVH_getDeviceLayout: invalid argument");
        return RT_ERR_INVALID;
    }
    if (d_nodes) *d_nodes = h->bvh8.nodes.p;
    if (num_nodes) *num_nodes = h->bvh8.num_nodes;
    if (d_tris) *d_tris = h->bvh8.tris.p;
    if (num_tris) *num_tris = h->bvh8.num_leaf_items;
    return RT_OK;
}

void cudaBVH_getBounds(CudaBVH_t h, float* cx, float* cy, float* cz, float* extent) {
    if (!h) return;
    if (cx) *cx = h->center[0];
    if (cy) *cy = h->center[1];
    if (cz) *cz = h->center[2];
    if (extent) *extent = h->extent;
}

int cudaBVH_getNumTris(CudaBVH_t h) { return h ? h->num_tris : 0; }
int cudaBVH_getNumCWBVHNodes(CudaBVH_t h) { return h ? h->bvh8.num_nodes : 0; }
int cudaBVH_getNumBVH4Nodes(CudaBVH_t h) {
    if (!h || !ensure_exports(h)) return 0;
    return h->num_bvh4;
}

const void* cudaBVH_getNodeData(CudaBVH_t h) {
    if (!h || !ensure_exports(h)) return nullptr;
    return h->h_bvh4.data();
}

void cudaBVH_getTriData(CudaBVH_t h, const float* outPtrs[9]) {
    if (!outPtrs) return;
    if (!h || !ensure_exports(h)) {
        for (int i = 0; i < 9; i++) outPtrs[i] = nullptr;
        return;
    }
    for (int i = 0; i < 9; i++) outPtrs[i] = h->h_soa[i].data();
}

int cudaBVH_getStacklessBVH2(CudaBVH_t h, uint32_t** outData) {
    if (!outData) return 0;
    if (!h || !ensure_exports(h)) {
        *outData = nullptr;
        return 0;
    }
    *outData = h->h_dfs.data();
    return (int)(h->h_dfs.size() / 8);
}

int cudaBVH_getPackedTris(CudaBVH_t h, float** outData) {
    if (!outData) return 0;
    if (!h || !ensure_exports(h)) {
        *outData = nullptr;
        return 0;
    }
    *outData = h->h_packed.data();
    return (int)(h->h_packed.size() / 4);
}

float cudaBVH_tracePrimary(CudaBVH_t h, int side, float camOx, float camOy, float camOz, float* outHitT) {
    if (!h || side <= 0 || side > 46340) {
        set_error("cudaBVH_tracePrimary: invalid argument");
        return 0.f;
    }
    const int n = side * side;
    std::lock_guard<std::mutex> g(h->mu);
    if (!h->stage_rays.ensure(n) || !h->stage_hits.ensure(n) || !h->stage_f.ensure(n)) return 0.f;
    launch_gen_square(h->stage_rays.p, side, camOx, camOy, camOz, 0);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int* work = next_counter(h->counters, h->counter_next, 0);
    cudaEventRecord(e0, 0);
    const int rc = launch_trace_blas(h->bvh8, h->stage_rays.p, n, h->stage_hits.p, nullptr, nullptr, work, h->status.p, 0);
    cudaEventRecord(e1, 0);
    float ms = 0.f;
    bool ok = rc == RT_OK && RT_CUDA(cudaEventSynchronize(e1));
    if (ok) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!ok) return 0.f;
    if (outHitT) {
        launch_hit_t(h->stage_hits.p, n, h->stage_f.p, 0);
        if (!RT_CUDA(cudaMemcpy(outHitT, h->stage_f.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost))) return 0.f;
    }
    if (check_status(h) != RT_OK) return 0.f;
    return ms > 0.f ? (float)n / (ms * 1000.f) : 0.f;
}

float cudaBVH_traceDiffuse(CudaBVH_t h, int n, const float* ox, const float* oy, const float* oz, const float* dx,
                           const float* dy, const float* dz, float* outHitT) {
    if (!h || n <= 0 || !ox || !oy || !oz || !dx || !dy || !dz) {
        set_error("cudaBVH_traceDiffuse: invalid argument");
        return 0.f;
    }
    std::lock_guard<std::mutex> g(h->mu);
    if (!h->stage_rays.ensure(n) || !h->stage_hits.ensure(n) || !h->stage_f.ensure((size_t)n * 6)) return 0.f;
    const float* src[6] = {ox, oy, oz, dx, dy, dz};
    for (int c = 0; c < 6; c++)
        if (!RT_CUDA(cudaMemcpyAsync(h->stage_f.p + (size_t)c * n, src[c], sizeof(float) * (size_t)n,
                                     cudaMemcpyHostToDevice, 0)))
            return 0.f;
    launch_soa_rays(h->stage_f.p, n, h->stage_rays.p, 0);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int* work = next_counter(h->counters, h->counter_next, 0);
    cudaEventRecord(e0, 0);
    const int rc = launch_trace_blas(h->bvh8, h->stage_rays.p, n, h->stage_hits.p, nullptr, nullptr, work, h->status.p, 0);
    cudaEventRecord(e1, 0);
    float ms = 0.f;
    bool ok = rc == RT_OK && RT_CUDA(cudaEventSynchronize(e1));
    if (ok) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!ok) return 0.f;
    if (outHitT) {
        launch_hit_t(h->stage_hits.p, n, h->stage_f.p, 0);
        if (!RT_CUDA(cudaMemcpy(outHitT, h->stage_f.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost))) return 0.f;
    }
    if (check_status(h) != RT_OK) return 0.f;
    return ms > 0.f ? (float)n / (ms * 1000.f) : 0.f;
}

int cudaBVH_traceToRGBA(CudaBVH_t h, int width, int height, float camOx, float camOy, float camOz,
                        uint32_t* outRGBA_host) {
    if (!h || width <= 0 || height <= 0 || !outRGBA_host) {
        set_error("cudaBVH_traceToRGBA: invalid argument");
        return -1;
    }
    std::lock_guard<std::mutex> g(h->mu);
    const size_t n = (size_t)width * height;
    if (!h->stage_f.ensure(n)) return -1;
    if (!render_rgba(h, width, height, camOx, camOy, camOz, h->stage_f.p, 0, 0)) return -1;
    return RT_CUDA(cudaMemcpy(outRGBA_host, h->stage_f.p, n * 4, cudaMemcpyDeviceToHost)) ? 0 : -1;
}

int cudaBVH_traceToGPUPtr(CudaBVH_t h, int width, int height, float camOx, float camOy, float camOz, void* d_out,
                          int outFmt) {
    if (!h || width <= 0 || height <= 0 || !d_out || outFmt < 0 || outFmt > 3) {
        set_error("cudaBVH_traceToGPUPtr: invalid argument");
        return -1;
    }
    std::lock_guard<std::mutex> g(h->mu);
    return render_rgba(h, width, height, camOx, camOy, camOz, d_out, outFmt, 0) ? 0 : -1;
}

void cudaBVH_traceToGPUAsync(CudaBVH_t h, int width, int height, float camOx, float camOy, float camOz, void* d_out,
                             int outFmt) {
    static std::atomic<int> calls{0};
    if (!h || width <= 0 || height <= 0 || !d_out || outFmt < 0 || outFmt > 3) {
        set_error("cudaBVH_traceToGPUAsync: invalid argument");
        return;
    }
    g_async.submit(h, width, height, camOx, camOy, camOz, outFmt, d_out, 0);
    if (calls.fetch_add(1) == 0) g_async.wait_first();
}

int cudaBVH_traceToHostPtr(CudaBVH_t h, int width, int height, float camOx, float camOy, float camOz, void* h_out,
                           int outFmt, uint64_t bufSize) {
    static std::atomic<int> calls{0};
    if (!h || width <= 0 || height <= 0 || !h_out || outFmt < 0 || outFmt > 3 || bufSize == 0) {
        set_error("cudaBVH_traceToHostPtr: invalid argument");
        return -1;
    }
    g_async.submit(h, width, height, camOx, camOy, camOz, outFmt, nullptr, bufSize);
    if (calls.fetch_add(1) == 0) g_async.wait_first();
    std::lock_guard<std::mutex> g(g_async.m);
    if (g_async.has_result && g_async.host[g_async.read_idx].size() >= bufSize)
        memcpy(h_out, g_async.host[g_async.read_idx].data(), bufSize);
    return 0;
}

void* cudaBVH_importBufferFd(int fd, uint64_t size) {
    if (fd < 0 || size == 0) {
        set_error("cudaBVH_importBufferFd: invalid argument");
        return nullptr;
    }
    cudaExternalMemoryHandleDesc desc;
    memset(&desc, 0, sizeof(desc));
    desc.type = cudaExternalMemoryHandleTypeOpaqueFd;
    desc.handle.fd = fd;
    desc.size = size;
    cudaExternalMemory_t ext;
    if (!RT_CUDA(cudaImportExternalMemory(&ext, &desc))) return nullptr;
    cudaExternalMemoryBufferDesc bd;
    memset(&bd, 0, sizeof(bd));
    bd.offset = 0;
    bd.size = size;
    void* p = nullptr;
    if (!RT_CUDA(cudaExternalMemoryGetMappedBuffer(&p, ext, &bd))) {
        cudaDestroyExternalMemory(ext);
        return nullptr;
    }
    return p;
}

int cudaBVH_readGPUMemoryFd(int fd, uint64_t allocationSize, uint64_t offset, uint64_t size, void* dst) {
    if (fd < 0 || !dst || size == 0 || offset + size > allocationSize) {
        set_error("cudaBVH_readGPUMemoryFd: invalid argument");
        return -1;
    }
    cudaExternalMemoryHandleDesc desc;
    memset(&desc, 0, sizeof(desc));
    desc.type = cudaExternalMemoryHandleTypeOpaqueFd;
    desc.handle.fd = fd;
    desc.size = allocationSize;
    cudaExternalMemory_t ext;
    if (!RT_CUDA(cudaImportExternalMemory(&ext, &desc))) return -1;
    cudaExternalMemoryBufferDesc bd;
    memset(&bd, 0, sizeof(bd));
    bd.offset = offset;
    bd.size = size;
    void* p = nullptr;
    int rc = -1;
    if (RT_CUDA(cudaExternalMemoryGetMappedBuffer(&p, ext, &bd))) {
        if (RT_CUDA(cudaMemcpy(dst, p, size, cudaMemcpyDeviceToHost))) rc = 0;
        cudaFree(p);
    }
    cudaDestroyExternalMemory(ext);
    return rc;
}

void cudaBVH_resetDevice(void) {
    cudaDeviceSynchronize();
    // the reset ends this context: the scratch address looked up in it is void
    noalloc_forget_current_device();
    cudaDeviceReset();
}

CudaBVH_t cudaBVH_buildFromAABBs(const float* aabbs, int numAABBs) {
    clear_error();
    if (!aabbs || numAABBs <= 0) {
        set_error("cudaBVH_buildFromAABBs: empty input");
        return nullptr;
    }
    // one triangle per AABB whose bounding box is the AABB, as the reference
    // does (layer/cuda_bvh_backend.cu:1597-1606), so leaf index = AABB index
    std::vector<CudaTri> t((size_t)numAABBs);
    for (int i = 0; i < numAABBs; i++) {
        const float* a = aabbs + (size_t)i * 6;
        t[i] = CudaTri{{a[0], a[1], a[2]}, {a[3], a[4], a[5]}, {a[3], a[1], a[2]}};
    }
    return cudaBVH_build(t.data(), numAABBs);
}

}  // extern "C"
