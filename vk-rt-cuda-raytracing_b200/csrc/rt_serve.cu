// rt_serve.cu -- the served form: a request loop over scenes resident in HBM.
//
// Scenes are copied once into one arena (8-wide nodes and triangle records
// of every scene back to back, child and triangle bases rebased), so a single
// kernel launch can trace rays of any mix of scenes.  Clients submit trace
// requests (scene, closest or any hit, a ray batch in host or device memory)
// from any thread; one scheduler thread runs the loop:
//
//   admit    host-buffer requests in arrival order while their footprint
//            (rays + results, 256-byte aligned) fits both the staging pool
//            and the HBM budget left after the resident scenes, and while
//            fewer than max_inflight requests are admitted; their rays are
//            copied host->device on the copy stream, oldest first, in
//            chunk-sized pieces that each record an event, with at most
//            prefetch_rays copied rays waiting for a wavefront;
//   batch    the rays whose copy has landed and that are not yet traced are
//            cut into chunks of at most chunk_rays and packed, oldest
//            request first, into a shared wavefront of at most wave_rays
//            rays: one persistent work-stealing launch per hit kind over a
//            segment table, so requests of different sizes and scenes share
//            the same warps;
//   overlap  up to max_waves wavefronts are in flight on their own streams:
//            a new wavefront's blocks fill the SMs as the previous one
//            drains, while admission copies of later requests proceed on
//            the copy stream and results of finished chunks go back
//            device->host on a third stream;
//   retire   a request completes when the results of all its chunks are
//            back; its staging memory returns to the pool at once, which is
//            what admits the next waiting request.
//
// Results do not depend on the mix: every ray's result is fixed by the
// triangle test and the (t, primitive) tie rule alone, whichever warp, launch
// or wavefront traces it.
//
// The reference has no served form; its per-call path (one synchronous trace
// call per ray batch, layer/cuda_bvh_backend.cu:526-598) is what this loop is
// measured against.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

#include "rt_internal.h"
#include "rt_legacy.h"
#include "rt_trace.cuh"

using namespace rtb;

namespace {

constexpr size_t kAlign = 256;

// A wavefront's segment table moves host->device and its status word
// device->host through the SMs, reading and writing the pinned staging
// directly: the copy engines carry request rays and results in large
// pieces, and a small copy queued behind them held each wavefront's launch
// (measured on the 256-request trace: trace streams busy 200+ ms of a
// 220 ms span while the kernels themselves needed far less).
__global__ void k_fetch_segs(const uint4* __restrict__ src, uint4* __restrict__ dst, int n16) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += gridDim.x * blockDim.x) dst[i] = src[i];
}
__global__ void k_put_status(const int* __restrict__ src, int* __restrict__ dst) { *dst = *src; }
constexpr int kMaxSeg = 512;  // segments per hit kind in one wavefront

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// First-fit allocator over one device range, free extents coalesced.
class Pool {
   public:
    void init(size_t bytes) {
        size_ = bytes;
        free_.clear();
        if (bytes) free_[0] = bytes;
        used_ = peak_ = 0;
    }
    bool alloc(size_t bytes, size_t* off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes;
            const size_t at = it->first + bytes;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t size() const { return size_; }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }

   private:
    std::map<size_t, size_t> free_;
    size_t size_ = 0, used_ = 0, peak_ = 0;
};

struct Scene {
    uint32_t root;  // arena node index of the scene's root
    uint32_t node_off, nodes, tri_off, tris;
};

struct Request {
    uint64_t ticket = 0;
    int scene = 0;
    bool any = false;
    bool host = true;
    const RtRay* h_rays = nullptr;  // host-buffer request
    void* h_out = nullptr;
    const RtRay* d_rays = nullptr;  // device rays (staged copy or the client's)
    void* d_out = nullptr;
    int n = 0;
    size_t pool_off = 0, pool_bytes = 0;
    int next_ray = 0;        // rays handed to wavefronts so far
    int ready_rays = 0;      // rays whose host->device copy has completed
    int issued_rays = 0;     // rays whose host->device copy has been issued
    std::vector<std::pair<int, cudaEvent_t>> pieces;  // (end ray, copy event) in copy order
    size_t pieces_ready = 0;
    int chunks_pending = 0;  // chunks in flight
    int waves = 0;
    int status = RT_OK;
    bool done = false;
    double t_submit = 0, t_admit = 0, t_done = 0;
};

struct Chunk {
    Request* req;
    int first, count;
};

struct WaveSlot {
    cudaStream_t stream = nullptr;
    cudaEvent_t traced = nullptr, done = nullptr;
    DevBuf<WaveSeg> d_segs;
    WaveSeg* h_segs = nullptr;  // pinned staging of the segment table
    int* h_status = nullptr;    // pinned status word of this wavefront
    // the same two pinned buffers as the device addresses them (mapped), or
    // null where the device cannot: then copy engines move them instead
    const uint4* m_segs = nullptr;
    int* m_status = nullptr;
    DevBuf<int> work;           // [0] closest, [1] any
    DevBuf<int> status;
    std::vector<Chunk> chunks;
    bool busy = false;
    uint64_t rays = 0;
};

}  // namespace

struct RtServerHandle {
    RtServerConfig cfg{};
    int device = 0;
    std::chrono::steady_clock::time_point t0;
    // resident scenes
    DevBuf<Bvh8Node> nodes;
    DevBuf<TriRec> tris;
    uint32_t nodes_used = 0, tris_used = 0;
    std::vector<Scene> scenes;
    // staging pool for host-buffer requests
    DevBuf<unsigned char> pool_mem;
    Pool pool;
    // streams
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    std::vector<cudaEvent_t> spare_events;
    std::vector<std::unique_ptr<WaveSlot>> slots;
    std::deque<WaveSlot*> inflight;  // in launch order
    // requests
    std::mutex mu;
    std::condition_variable cv_submit, cv_done;
    std::deque<Request*> submitted;  // guarded by mu
    std::unordered_map<uint64_t, std::unique_ptr<Request>> all;  // guarded by mu
    uint64_t next_ticket = 1;
    std::deque<Request*> waiting;  // scheduler-owned: not yet admitted
    std::deque<Request*> staged;   // scheduler-owned: admitted, rays left to trace
    std::deque<Request*> to_copy;  // scheduler-owned: admitted, copies left to issue
    int64_t pending_rays = 0;      // copies issued whose rays are not yet in a wavefront
    int admitted = 0;
    // scene additions run on the scheduler thread between wavefronts
    struct SceneJob {
        CudaBVH_t bvh;
        int result;
        bool finished;
    };
    std::deque<SceneJob*> scene_jobs;  // guarded by mu
    // stats
    std::atomic<uint64_t> req_done{0}, rays_done{0}, waves{0};
    std::atomic<bool> stop{false};
    std::thread th;
    std::string fatal;

    double now_us() const {
        return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
    }
    size_t resident_bytes() const { return nodes.bytes() + tris.bytes(); }

    cudaEvent_t get_event() {
        if (!spare_events.empty()) {
            cudaEvent_t e = spare_events.back();
            spare_events.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        return RT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)) ? e : nullptr;
    }
    void update_ready(Request* r) {
        while (r->pieces_ready < r->pieces.size()) {
            const cudaError_t q = cudaEventQuery(r->pieces[r->pieces_ready].second);
            if (q == cudaErrorNotReady) break;
            if (q != cudaSuccess) {
                cuda_ok(q, "request copy");
                r->status = RT_ERR_CUDA;
            }
            r->ready_rays = r->pieces[r->pieces_ready].first;
            r->pieces_ready++;
        }
    }
    void loop();
    int add_scene(CudaBVH_t b);
    void admit();
    void issue_copies();
    bool launch_wave(WaveSlot* w);
    bool retire();
    void complete(Request* r);
    void fail_all(const char* why);
};

int RtServerHandle::add_scene(CudaBVH_t b) {
    const Bvh8Device& src = b->bvh8;
    const uint32_t nn = (uint32_t)src.num_nodes, nt = (uint32_t)src.num_leaf_items;
    const size_t need_nodes = (size_t)nodes_used + nn, need_tris = (size_t)tris_used + nt;
    if (need_nodes >= 0xFFFFFFF0u || need_tris >= 0x7FFFFFF0u) {
        set_error("rtServer_addScene: arena index range exceeded");
        return RT_ERR_CAPACITY;
    }
    // grow the arena (no wavefront is in flight while this runs)
    const size_t want_nodes = std::max(need_nodes, nodes.n), want_tris = std::max(need_tris, tris.n);
    const size_t grow = (want_nodes - nodes.n) * sizeof(Bvh8Node) + (want_tris - tris.n) * sizeof(TriRec);
    if (resident_bytes() + grow + pool.used() > cfg.hbm_budget_bytes) {
        set_error("rtServer_addScene: HBM budget exceeded (%zu resident + %zu new > %llu)", resident_bytes(), grow,
                  (unsigned long long)cfg.hbm_budget_bytes);
        return RT_ERR_CAPACITY;
    }
    if (want_nodes > nodes.n) {
        DevBuf<Bvh8Node> nb;
        if (!nb.alloc(want_nodes)) return RT_ERR_NOMEM;
        if (nodes_used && !RT_CUDA(cudaMemcpyAsync(nb.p, nodes.p, (size_t)nodes_used * sizeof(Bvh8Node),
                                                   cudaMemcpyDeviceToDevice, copy_in)))
            return RT_ERR_CUDA;
        if (!RT_CUDA(cudaStreamSynchronize(copy_in))) return RT_ERR_CUDA;
        std::swap(nodes.p, nb.p);
        std::swap(nodes.n, nb.n);
    }
    if (want_tris > tris.n) {
        DevBuf<TriRec> nb;
        if (!nb.alloc(want_tris)) return RT_ERR_NOMEM;
        if (tris_used && !RT_CUDA(cudaMemcpyAsync(nb.p, tris.p, (size_t)tris_used * sizeof(TriRec),
                                                  cudaMemcpyDeviceToDevice, copy_in)))
            return RT_ERR_CUDA;
        if (!RT_CUDA(cudaStreamSynchronize(copy_in))) return RT_ERR_CUDA;
        std::swap(tris.p, nb.p);
        std::swap(tris.n, nb.n);
    }
    launch_rebase_nodes(src.nodes.p, nodes.p + nodes_used, (int)nn, nodes_used, tris_used, copy_in);
    if (nt && !RT_CUDA(cudaMemcpyAsync(tris.p + tris_used, src.tris.p, (size_t)nt * sizeof(TriRec),
                                       cudaMemcpyDeviceToDevice, copy_in)))
        return RT_ERR_CUDA;
    if (!RT_CUDA(cudaStreamSynchronize(copy_in))) return RT_ERR_CUDA;
    Scene sc{nodes_used, nodes_used, nn, tris_used, nt};
    nodes_used += nn;
    tris_used += nt;
    std::lock_guard<std::mutex> g(mu);  // submit() reads the scene count
    scenes.push_back(sc);
    return (int)scenes.size() - 1;
}

void RtServerHandle::complete(Request* r) {
    r->t_done = now_us();
    for (auto& pc : r->pieces) spare_events.push_back(pc.second);
    r->pieces.clear();
    if (r->host && r->pool_bytes) {
        pool.release(r->pool_off, r->pool_bytes);
        r->pool_bytes = 0;
    }
    admitted--;
    req_done++;
    rays_done += (uint64_t)r->n;
    {
        std::lock_guard<std::mutex> g(mu);
        r->done = true;
    }
    cv_done.notify_all();
}

void RtServerHandle::fail_all(const char* why) {
    const std::string detail = rtGetLastError();  // this thread's last CUDA error, if any
    std::lock_guard<std::mutex> g(mu);
    fatal = detail.empty() ? std::string(why) : std::string(why) + ": " + detail;
    for (auto& kv : all) {
        if (!kv.second->done) {
            kv.second->status = RT_ERR_CUDA;
            kv.second->done = true;
            kv.second->t_done = now_us();
        }
    }
    submitted.clear();
    waiting.clear();
    staged.clear();
    to_copy.clear();
    cv_done.notify_all();
}

// Issues host->device copies of admitted requests in chunk-sized pieces,
// oldest first, each recording an event, while fewer than prefetch_rays
// copied rays wait for a wavefront.  The read-ahead bound keeps completions
// in arrival order: copies of later requests do not take PCIe bandwidth from
// the results of earlier ones.
void RtServerHandle::issue_copies() {
    while (!to_copy.empty() && pending_rays < cfg.prefetch_rays) {
        Request* r = to_copy.front();
        const int b = r->issued_rays, e = std::min(r->n, b + cfg.chunk_rays);
        cudaEvent_t ev = get_event();
        if (!ev || !RT_CUDA(cudaMemcpyAsync((void*)(r->d_rays + b), r->h_rays + b, (size_t)(e - b) * sizeof(RtRay),
                                            cudaMemcpyHostToDevice, copy_in)) ||
            !RT_CUDA(cudaEventRecord(ev, copy_in))) {
            if (ev) spare_events.push_back(ev);
            fail_all("request copy could not be issued");
            stop = true;
            return;
        }
        r->pieces.push_back({e, ev});
        pending_rays += e - b;
        r->issued_rays = e;
        if (e == r->n) to_copy.pop_front();
    }
}

void RtServerHandle::admit() {
    while (!waiting.empty() && admitted < cfg.max_inflight) {
        Request* r = waiting.front();
        if (r->host && r->n > 0) {
            const size_t ob = r->any ? (size_t)r->n : (size_t)r->n * sizeof(RtHit);
            const size_t fp = align_up((size_t)r->n * sizeof(RtRay)) + align_up(ob);
            size_t off = 0;
            if (resident_bytes() + pool.used() + fp > cfg.hbm_budget_bytes || !pool.alloc(fp, &off)) break;
            r->pool_off = off;
            r->pool_bytes = fp;
            unsigned char* base = pool_mem.p + off;
            r->d_rays = reinterpret_cast<const RtRay*>(base);
            r->d_out = base + align_up((size_t)r->n * sizeof(RtRay));
            to_copy.push_back(r);
        } else {
            r->ready_rays = r->n;
        }
        waiting.pop_front();
        admitted++;
        r->t_admit = now_us();
        staged.push_back(r);
    }
}

bool RtServerHandle::launch_wave(WaveSlot* w) {
    w->chunks.clear();
    w->rays = 0;
    int nc = 0, na = 0;
    uint32_t tc = 0, ta = 0;
    const uint32_t cap = (uint32_t)cfg.wave_rays;
    for (auto it = staged.begin(); it != staged.end() && tc + ta < cap;) {
        Request* r = *it;
        update_ready(r);
        int& ns = r->any ? na : nc;
        uint32_t& tk = r->any ? ta : tc;
        while (r->next_ray < r->ready_rays && tc + ta < cap && ns < kMaxSeg) {
            const int cnt = (int)std::min<uint32_t>(
                {(uint32_t)cfg.chunk_rays, (uint32_t)(r->ready_rays - r->next_ray), cap - tc - ta});
            WaveSeg& sg = w->h_segs[(r->any ? kMaxSeg : 0) + ns];
            sg.rays = r->d_rays + r->next_ray;
            sg.out = r->any ? (void*)((uint8_t*)r->d_out + r->next_ray)
                            : (void*)((RtHit*)r->d_out + r->next_ray);
            sg.first = tk;
            sg.root = scenes[r->scene].root;
            sg.pad[0] = sg.pad[1] = 0;
            w->chunks.push_back({r, r->next_ray, cnt});
            if (r->host) pending_rays -= cnt;
            r->next_ray += cnt;
            r->chunks_pending++;
            ns++;
            tk += (uint32_t)cnt;
        }
        if (r->next_ray >= r->n) it = staged.erase(it);
        else ++it;
        if (ns >= kMaxSeg) break;
    }
    if (w->chunks.empty()) return false;
    for (const Chunk& c : w->chunks) c.req->waves++;
    w->rays = tc + ta;
    cudaStream_t s = w->stream;
    bool ok = true;
    if (w->m_segs) {
        static_assert(sizeof(WaveSeg) % 16 == 0, "segment table moves as 16-byte words");
        k_fetch_segs<<<8, 256, 0, s>>>(w->m_segs, reinterpret_cast<uint4*>(w->d_segs.p),
                                       (int)(sizeof(WaveSeg) * 2 * kMaxSeg / 16));
        ok = RT_CUDA(cudaGetLastError());
    } else {
        ok = RT_CUDA(cudaMemcpyAsync(w->d_segs.p, w->h_segs, sizeof(WaveSeg) * 2 * kMaxSeg, cudaMemcpyHostToDevice, s));
    }
    ok = ok && RT_CUDA(cudaMemsetAsync(w->work.p, 0, 2 * sizeof(int), s)) &&
              RT_CUDA(cudaMemsetAsync(w->status.p, 0, sizeof(int), s));
    const uint4* nd = reinterpret_cast<const uint4*>(nodes.p);
    const float4* tr = reinterpret_cast<const float4*>(tris.p);
    if (ok && nc) ok = launch_trace_wave(nd, tr, w->d_segs.p, nc, (int)tc, false, w->work.p, w->status.p,
                                         TRACE_MINB, s) == RT_OK;
    if (ok && na) ok = launch_trace_wave(nd, tr, w->d_segs.p + kMaxSeg, na, (int)ta, true, w->work.p + 1,
                                         w->status.p, TRACE_MINB_ANY, s) == RT_OK;
    if (ok && w->m_status) {
        k_put_status<<<1, 1, 0, s>>>(w->status.p, w->m_status);
        ok = RT_CUDA(cudaGetLastError());
    } else if (ok) {
        ok = RT_CUDA(cudaMemcpyAsync(w->h_status, w->status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    ok = ok && RT_CUDA(cudaEventRecord(w->traced, s)) && RT_CUDA(cudaStreamWaitEvent(copy_out, w->traced, 0));
    for (const Chunk& c : w->chunks) {
        if (!ok) break;
        Request* r = c.req;
        if (!r->host) continue;
        const size_t es = r->any ? 1 : sizeof(RtHit);
        ok = RT_CUDA(cudaMemcpyAsync((char*)r->h_out + (size_t)c.first * es, (const char*)r->d_out + (size_t)c.first * es,
                                     (size_t)c.count * es, cudaMemcpyDeviceToHost, copy_out));
    }
    ok = ok && RT_CUDA(cudaEventRecord(w->done, copy_out));
    w->busy = true;
    inflight.push_back(w);
    waves++;
    return ok;
}

// Retires the oldest wavefront if its results are back; true if it did.
bool RtServerHandle::retire() {
    if (inflight.empty()) return false;
    WaveSlot* w = inflight.front();
    const cudaError_t q = cudaEventQuery(w->done);
    if (q == cudaErrorNotReady) return false;
    if (q != cudaSuccess) {
        cuda_ok(q, "wavefront");
        fail_all("CUDA error in a wavefront");
        stop = true;
        return false;
    }
    inflight.pop_front();
    const int st = *w->h_status;
    for (const Chunk& c : w->chunks) {
        Request* r = c.req;
        if (st & RT_STATUS_STACK) r->status = RT_ERR_STACK;
        if (--r->chunks_pending == 0 && r->next_ray >= r->n) complete(r);
    }
    w->chunks.clear();
    w->busy = false;
    return true;
}

void RtServerHandle::loop() {
    cudaSetDevice(device);
    for (;;) {
        // take new submissions and scene jobs
        std::deque<SceneJob*> jobs;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (stop && submitted.empty() && waiting.empty() && staged.empty() && inflight.empty() &&
                scene_jobs.empty())
                break;
            if (submitted.empty() && waiting.empty() && staged.empty() && inflight.empty() && scene_jobs.empty())
                cv_submit.wait_for(lk, std::chrono::milliseconds(2));
            while (!submitted.empty()) {
                waiting.push_back(submitted.front());
                submitted.pop_front();
            }
            if (inflight.empty()) jobs.swap(scene_jobs);
        }
        for (SceneJob* j : jobs) {
            const int rc = add_scene(j->bvh);
            {
                std::lock_guard<std::mutex> g(mu);
                j->result = rc;
                j->finished = true;
            }
            cv_done.notify_all();
        }
        bool progress = false;
        while (retire()) progress = true;
        if (stop && !fatal.empty()) break;
        admit();
        issue_copies();
        bool scene_pending;
        {
            std::lock_guard<std::mutex> g(mu);
            scene_pending = !scene_jobs.empty();
        }
        // zero-ray requests complete at admission
        for (auto it = staged.begin(); it != staged.end();) {
            Request* r = *it;
            if (r->n == 0) {
                it = staged.erase(it);
                complete(r);
                progress = true;
            } else {
                ++it;
            }
        }
        while (!scene_pending && !staged.empty() && (int)inflight.size() < cfg.max_waves) {
            WaveSlot* w = nullptr;
            for (auto& s : slots)
                if (!s->busy) {
                    w = s.get();
                    break;
                }
            if (!w) break;
            if (!launch_wave(w)) {
                if (!w->busy) break;
                fail_all("wavefront launch failed");
                stop = true;
                break;
            }
            progress = true;
        }
        issue_copies();
        if (!progress) std::this_thread::yield();
    }
    cudaStreamSynchronize(copy_out);
}

extern "C" {

RtServer_t rtServer_create(const RtServerConfig* cfg_in) {
    clear_error();
    RtServerConfig c{};
    if (cfg_in) c = *cfg_in;
    if (!c.hbm_budget_bytes) c.hbm_budget_bytes = 120ull << 30;
    if (!c.pool_bytes) c.pool_bytes = 4ull << 30;
    if (c.max_inflight <= 0) c.max_inflight = 256;
    if (c.wave_rays <= 0) c.wave_rays = 4 << 20;
    if (c.chunk_rays <= 0) c.chunk_rays = 1 << 20;
    if (c.max_waves <= 0) c.max_waves = 2;
    if (c.prefetch_rays <= 0) c.prefetch_rays = 2 * c.wave_rays;
    if (c.max_waves > 8 || c.chunk_rays > c.wave_rays || c.pool_bytes > c.hbm_budget_bytes) {
        set_error("rtServer_create: invalid configuration");
        return nullptr;
    }
    std::unique_ptr<RtServerHandle> s(new (std::nothrow) RtServerHandle());
    if (!s) return nullptr;
    s->cfg = c;
    s->t0 = std::chrono::steady_clock::now();
    cudaGetDevice(&s->device);
    bool ok = s->pool_mem.alloc(c.pool_bytes) &&
              RT_CUDA(cudaStreamCreateWithFlags(&s->copy_in, cudaStreamNonBlocking)) &&
              RT_CUDA(cudaStreamCreateWithFlags(&s->copy_out, cudaStreamNonBlocking));
    s->pool.init(c.pool_bytes);
    for (int i = 0; ok && i < c.max_waves; i++) {
        auto w = std::make_unique<WaveSlot>();
        ok = RT_CUDA(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking)) &&
             RT_CUDA(cudaEventCreateWithFlags(&w->traced, cudaEventDisableTiming)) &&
             RT_CUDA(cudaEventCreateWithFlags(&w->done, cudaEventDisableTiming)) && w->d_segs.alloc(2 * kMaxSeg) &&
             w->work.alloc(2) && w->status.alloc(1) &&
             RT_CUDA(cudaMallocHost(&w->h_segs, sizeof(WaveSeg) * 2 * kMaxSeg)) &&
             RT_CUDA(cudaMallocHost(&w->h_status, sizeof(int)));
        if (ok) {  // device addresses of the pinned staging (unified addressing maps it)
            void *ds = nullptr, *dst = nullptr;
            if (cudaHostGetDevicePointer(&ds, w->h_segs, 0) == cudaSuccess &&
                cudaHostGetDevicePointer(&dst, w->h_status, 0) == cudaSuccess && ds && dst &&
                reinterpret_cast<uintptr_t>(ds) % 16 == 0) {
                w->m_segs = static_cast<const uint4*>(ds);
                w->m_status = static_cast<int*>(dst);
            } else {
                cudaGetLastError();
            }
        }
        s->slots.push_back(std::move(w));
    }
    if (!ok) {
        rtServer_destroy(s.release());
        return nullptr;
    }
    RtServerHandle* h = s.release();
    h->th = std::thread([h] { h->loop(); });
    return h;
}

int rtServer_addScene(RtServer_t s, CudaBVH_t bvh) {
    clear_error();
    if (!s || !bvh) {
        set_error("rtServer_addScene: invalid argument");
        return RT_ERR_INVALID;
    }
    RtServerHandle::SceneJob job{bvh, 0, false};
    std::unique_lock<std::mutex> lk(s->mu);
    if (!s->fatal.empty()) {
        set_error("rtServer_addScene: server failed: %s", s->fatal.c_str());
        return RT_ERR_CUDA;
    }
    s->scene_jobs.push_back(&job);
    s->cv_submit.notify_one();
    s->cv_done.wait(lk, [&] { return job.finished; });
    return job.result;
}

static int submit(RtServer_t s, int scene, int any_hit, const RtRay* rays, int n, void* out, bool host,
                  uint64_t* ticket) {
    clear_error();
    if (!s || !ticket || n < 0 || (n > 0 && (!rays || !out))) {
        set_error("rtServer_submit: invalid argument");
        return RT_ERR_INVALID;
    }
    if (!host && !check_aligned("rtServer_submitDevice", rays, out, any_hit ? 1 : 16)) return RT_ERR_INVALID;
    std::unique_ptr<Request> r(new Request());
    r->scene = scene;
    r->any = any_hit != 0;
    r->host = host;
    r->n = n;
    if (host) {
        r->h_rays = rays;
        r->h_out = out;
        const size_t ob = r->any ? (size_t)n : (size_t)n * sizeof(RtHit);
        const size_t fp = align_up((size_t)n * sizeof(RtRay)) + align_up(ob);
        if (fp > s->pool.size()) {
            set_error("rtServer_submit: request footprint %zu bytes exceeds the staging pool (%zu)", fp,
                      s->pool.size());
            return RT_ERR_CAPACITY;
        }
    } else {
        r->d_rays = rays;
        r->d_out = out;
    }
    std::lock_guard<std::mutex> g(s->mu);
    if (!s->fatal.empty()) {
        set_error("rtServer_submit: server failed: %s", s->fatal.c_str());
        return RT_ERR_CUDA;
    }
    if (scene < 0 || scene >= (int)s->scenes.size()) {
        set_error("rtServer_submit: no scene %d", scene);
        return RT_ERR_INVALID;
    }
    r->ticket = s->next_ticket++;
    r->t_submit = s->now_us();
    *ticket = r->ticket;
    s->submitted.push_back(r.get());
    s->all[r->ticket] = std::move(r);
    s->cv_submit.notify_one();
    return RT_OK;
}

int rtServer_submit(RtServer_t s, int scene, int any_hit, const RtRay* h_rays, int n, void* h_out,
                    uint64_t* ticket) {
    return submit(s, scene, any_hit, h_rays, n, h_out, true, ticket);
}

int rtServer_submitDevice(RtServer_t s, int scene, int any_hit, const RtRay* d_rays, int n, void* d_out,
                          uint64_t* ticket) {
    return submit(s, scene, any_hit, d_rays, n, d_out, false, ticket);
}

int rtServer_wait(RtServer_t s, uint64_t ticket, int timeout_ms, RtRequestInfo* info) {
    clear_error();
    if (!s) {
        set_error("rtServer_wait: invalid argument");
        return RT_ERR_INVALID;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) {
        set_error("rtServer_wait: unknown ticket %llu", (unsigned long long)ticket);
        return RT_ERR_INVALID;
    }
    Request* r = it->second.get();
    const auto pred = [&] { return r->done; };
    if (timeout_ms < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
        set_error("rtServer_wait: ticket %llu not done within %d ms", (unsigned long long)ticket, timeout_ms);
        return RT_ERR_TIMEOUT;
    }
    const int st = r->status;
    if (info) {
        info->submit_us = r->t_submit;
        info->admit_us = r->t_admit;
        info->done_us = r->t_done;
        info->status = st;
        info->waves = r->waves;
    }
    s->all.erase(it);
    if (st != RT_OK) set_error("rtServer_wait: request failed (%d)%s%s", st, s->fatal.empty() ? "" : ": ",
                               s->fatal.c_str());
    return st;
}

int rtServer_getStats(RtServer_t s, RtServerStats* st) {
    if (!s || !st) {
        set_error("rtServer_getStats: invalid argument");
        return RT_ERR_INVALID;
    }
    std::lock_guard<std::mutex> g(s->mu);
    st->requests_done = s->req_done;
    st->rays_done = s->rays_done;
    st->waves = s->waves;
    st->resident_bytes = s->resident_bytes();
    st->pool_bytes = s->pool.size();
    st->peak_pool_used = s->pool.peak();
    st->num_scenes = (int)s->scenes.size();
    return RT_OK;
}

void rtServer_destroy(RtServer_t s) {
    if (!s) return;
    if (s->th.joinable()) {
        {
            std::lock_guard<std::mutex> g(s->mu);
            s->stop = true;
        }
        s->cv_submit.notify_all();
        s->th.join();
    }
    for (auto& w : s->slots) {
        if (w->stream) cudaStreamSynchronize(w->stream);
        if (w->stream) cudaStreamDestroy(w->stream);
        if (w->traced) cudaEventDestroy(w->traced);
        if (w->done) cudaEventDestroy(w->done);
        if (w->h_segs) cudaFreeHost(w->h_segs);
        if (w->h_status) cudaFreeHost(w->h_status);
    }
    if (s->copy_in) cudaStreamSynchronize(s->copy_in);
    if (s->copy_out) cudaStreamSynchronize(s->copy_out);
    if (s->copy_in) cudaStreamDestroy(s->copy_in);
    if (s->copy_out) cudaStreamDestroy(s->copy_out);
    for (cudaEvent_t e : s->spare_events) cudaEventDestroy(e);
    for (auto& kv : s->all)
        for (auto& pc : kv.second->pieces) cudaEventDestroy(pc.second);
    delete s;
}

}  // extern "C"
