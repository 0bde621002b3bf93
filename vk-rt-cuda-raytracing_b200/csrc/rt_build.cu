// rt_build.cu -- GPU SAH builder of the binary BVH (the 8-wide collapse is
// in rt_collapse.cu).
//
// Replaces the reference's single-threaded CPU BVH2Builder
// (layer/cuda_bvh_backend.cu:201-251 / cuda_rt_v40.cu:790-840).  Cost model
// C = N_L*A(L) + N_R*A(R), the reference's split search; leaves at
// <= max_leaf primitives; depth >= max_sah_depth -> object-median split.
// Three tiers by task size, every step deterministic:
//   * tasks > small_task (1024) primitives: level-synchronous over all
//     tasks (and all scenes of a batch) at once.  Chunked CTA binning into
//     shared-memory bins (3 axes x 32 bins, count + box per bin, order-
//     independent atomics; a thread's run of primitives in one bin is
//     merged in registers first), one warp per task scans the 31 planes per
//     axis (lane = bin), a stable partition by chunk scans that also gathers
//     the children's centroid bounds.  The loop is queued ahead of the host:
//     counts stay on the device and the host reads each level's task count
//     one level late, so the GPU never waits for it.
//   * tasks of 33..small_task primitives: one CTA per task, node by node, in
//     shared memory (binned SAH, single-scan partition, child boxes from the
//     split's bins).
//   * subtrees of <= 32 primitives: one warp per subtree, exact SAH sweep
//     over centroid-sorted orders, a whole level per pass (k_build_warp).
// Scratch comes from the pooled stream-ordered allocator (TmpBuf).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>

#include "rt_internal.h"

namespace rtb {

constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr int CHUNK = 2048;          // primitives per binning CTA
constexpr int CHUNK_T = 256;         // threads per binning CTA
constexpr int SMALL_T = 128;         // threads per small-task CTA
constexpr int SMALL_STACK = 96;

// ---------------------------------------------------------------- scan --
template <int T>
__device__ int block_exclusive_scan(int v, int* ws, int& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < T / 32 ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(FULL, s, o);
            if (lane >= o) s += y;
        }
        if (lane < T / 32) ws[lane] = s;
    }
    __syncthreads();
    const int before = w ? ws[w - 1] : 0;
    total = ws[T / 32 - 1];
    __syncthreads();
    return before + x - v;
}

constexpr int SCAN_T = 256, SCAN_IPT = 8, SCAN_TILE = SCAN_T * SCAN_IPT;

__global__ void __launch_bounds__(SCAN_T) k_scan_tiles(const int* __restrict__ in, int* __restrict__ out, int n,
                                                       int* __restrict__ tile_sums) {
    __shared__ int ws[SCAN_T / 32];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_IPT;
    int v[SCAN_IPT];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; k++) {
        v[k] = base + k < n ? in[base + k] : 0;
        sum += v[k];
    }
    int total;
    int run = block_exclusive_scan<SCAN_T>(sum, ws, total);
#pragma unroll
    for (int k = 0; k < SCAN_IPT; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(int* __restrict__ out, int n, const int* __restrict__ tile_off) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tile_off[i / SCAN_TILE];
}

__global__ void k_scan_total(const int* __restrict__ in, const int* __restrict__ out, int n, int* total) {
    *total = n > 0 ? out[n - 1] + in[n - 1] : 0;
}

bool scan_exclusive(const int* d_in, int* d_out, int n, int* d_total, cudaStream_t s) {
    if (n <= 0) {
        if (d_total) cudaMemsetAsync(d_total, 0, sizeof(int), s);
        return true;
    }
    const int tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles == 1) {
        k_scan_tiles<<<1, SCAN_T, 0, s>>>(d_in, d_out, n, nullptr);
    } else {
        TmpBuf<int> sums;
        if (!sums.alloc((size_t)tiles * 2, s)) return false;
        int* offs = sums.p + tiles;
        k_scan_tiles<<<tiles, SCAN_T, 0, s>>>(d_in, d_out, n, sums.p);
        if (!scan_exclusive(sums.p, offs, tiles, nullptr, s)) return false;
        k_scan_add<<<(n + 255) / 256, 256, 0, s>>>(d_out, n, offs);
    }
    if (d_total) k_scan_total<<<1, 1, 0, s>>>(d_in, d_out, n, d_total);
    return RT_CUDA(cudaGetLastError());
}

// The same exclusive scan with its element count read on the device (d_n;
// null: all `cap` elements) and caller-provided scratch (scan_scratch_ints),
// so it can be enqueued into a graph whose counts the host never sees.
// Tiles past the count write a zero tile sum, so the next level's scan over
// all tiles stays exact.
__device__ __forceinline__ int scan_count(const int* d_n, int cap) { return d_n ? min(max(*d_n, 0), cap) : cap; }

__global__ void __launch_bounds__(SCAN_T) k_scan_tiles_n(const int* __restrict__ in, int* __restrict__ out, int cap,
                                                         const int* __restrict__ d_n, int* __restrict__ tile_sums) {
    __shared__ int ws[SCAN_T / 32];
    const int n = scan_count(d_n, cap);
    if (blockIdx.x * SCAN_TILE >= n) {  // block-uniform
        if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = 0;
        return;
    }
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_IPT;
    int v[SCAN_IPT];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; k++) {
        v[k] = base + k < n ? in[base + k] : 0;
        sum += v[k];
    }
    int total;
    int run = block_exclusive_scan<SCAN_T>(sum, ws, total);
#pragma unroll
    for (int k = 0; k < SCAN_IPT; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_add_n(int* __restrict__ out, int cap, const int* __restrict__ d_n,
                             const int* __restrict__ tile_off) {
    const int n = scan_count(d_n, cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] += tile_off[i / SCAN_TILE];
}

__global__ void k_scan_total_n(const int* __restrict__ in, const int* __restrict__ out, int cap,
                               const int* __restrict__ d_n, int* __restrict__ total) {
    const int n = scan_count(d_n, cap);
    *total = n > 0 ? out[n - 1] + in[n - 1] : 0;
}

size_t scan_scratch_ints(int cap) {
    size_t total = 1;
    for (int m = cap; m > SCAN_TILE;) {
        const int tiles = (m + SCAN_TILE - 1) / SCAN_TILE;
        total += 2 * (size_t)tiles;
        m = tiles;
    }
    return total;
}

bool scan_exclusive_dev(const int* d_in, int* d_out, int cap, const int* d_n, int* d_total, int* scratch,
                        cudaStream_t s) {
    if (cap > 0) {
        const int tiles = (cap + SCAN_TILE - 1) / SCAN_TILE;
        if (tiles == 1) {
            k_scan_tiles_n<<<1, SCAN_T, 0, s>>>(d_in, d_out, cap, d_n, nullptr);
        } else {
            int* sums = scratch;
            int* offs = scratch + tiles;
            k_scan_tiles_n<<<tiles, SCAN_T, 0, s>>>(d_in, d_out, cap, d_n, sums);
            if (!scan_exclusive_dev(sums, offs, tiles, nullptr, nullptr, scratch + 2 * tiles, s)) return false;
            k_scan_add_n<<<std::min((cap + 255) / 256, num_sms() * 16), 256, 0, s>>>(d_out, cap, d_n, offs);
        }
    }
    if (d_total) k_scan_total_n<<<1, 1, 0, s>>>(d_in, d_out, cap > 0 ? cap : 0, cap > 0 ? d_n : nullptr, d_total);
    return RT_CUDA(cudaGetLastError());
}

// Creates a conditional handle on the graph being captured on cs (value 0
// at every launch until a kernel sets it).
bool capture_conditional_handle(cudaStream_t cs, cudaGraphConditionalHandle* h) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    if (!RT_CUDA(cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, nullptr, nullptr))) return false;
    if (st != cudaStreamCaptureStatusActive || !g) {
        set_error("graph build: stream is not capturing");
        return false;
    }
    return RT_CUDA(cudaGraphConditionalHandleCreate(h, g, 0, cudaGraphCondAssignDefault));
}

// Appends a WHILE node on handle h at the capture position of cs; its body
// graph (empty, to be captured) is returned in *body.
bool capture_while(cudaStream_t cs, cudaGraphConditionalHandle h, cudaGraph_t* body) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    if (!RT_CUDA(cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &nd))) return false;
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    if (!RT_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p)) ||
        !RT_CUDA(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies)))
        return false;
    *body = p.conditional.phGraph_out[0];
    return true;
}

// -------------------------------------------------------- prim bounds --
__global__ void k_tri_bounds(const float* __restrict__ t9, int n, float4* __restrict__ lo,
                             float4* __restrict__ hi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* t = t9 + (size_t)i * 9;
    lo[i] = make_float4(fminf(fminf(t[0], t[3]), t[6]), fminf(fminf(t[1], t[4]), t[7]),
                        fminf(fminf(t[2], t[5]), t[8]), 0.f);
    hi[i] = make_float4(fmaxf(fmaxf(t[0], t[3]), t[6]), fmaxf(fmaxf(t[1], t[4]), t[7]),
                        fmaxf(fmaxf(t[2], t[5]), t[8]), 0.f);
}

void launch_tri_bounds(const float* d_tris9, int n, float4* d_lo, float4* d_hi, cudaStream_t s) {
    if (n > 0) k_tri_bounds<<<(n + 255) / 256, 256, 0, s>>>(d_tris9, n, d_lo, d_hi);
}

__device__ __forceinline__ float centroid(float lo, float hi) { return (lo + hi) * 0.5f; }
__device__ __forceinline__ float half_area(float lx, float ly, float lz, float hx, float hy, float hz) {
    const float dx = hx - lx, dy = hy - ly, dz = hz - lz;
    return dx * dy + dy * dz + dz * dx;
}
__device__ __forceinline__ int bin_of(float c, float cmin, float k) {
    int b = (int)((c - cmin) * k);
    return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
}
__device__ __forceinline__ float bin_scale(float cmin, float cmax) {
    const float ext = cmax - cmin;
    return ext > 0.f ? (float)kBins / ext : 0.f;
}

// Per-segment box and centroid box (12 ordered uints per segment); grid.y
// is the segment (so at most kMaxSegments of them), grid.x strides over its
// primitives.
constexpr int kMaxSegments = 65535;
__global__ void k_seg_bounds(const float4* __restrict__ lo, const float4* __restrict__ hi,
                             const int* __restrict__ seg_off, uint32_t* __restrict__ acc) {
    const int sgi = blockIdx.y;
    const int beg = seg_off[sgi], end = seg_off[sgi + 1];
    float b[12];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        b[k] = FLT_MAX; b[3 + k] = -FLT_MAX; b[6 + k] = FLT_MAX; b[9 + k] = -FLT_MAX;
    }
    for (int i = beg + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
        const float4 l = lo[i], h = hi[i];
        const float L[3] = {l.x, l.y, l.z}, H[3] = {h.x, h.y, h.z};
#pragma unroll
        for (int k = 0; k < 3; k++) {
            b[k] = fminf(b[k], L[k]);
            b[3 + k] = fmaxf(b[3 + k], H[k]);
            const float c = centroid(L[k], H[k]);
            b[6 + k] = fminf(b[6 + k], c);
            b[9 + k] = fmaxf(b[9 + k], c);
        }
    }
    uint32_t* a = acc + (size_t)sgi * 12;
#pragma unroll
    for (int k = 0; k < 12; k++) {
        const bool mx = (k >= 3 && k < 6) || k >= 9;
        float v = b[k];
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const float y = __shfl_xor_sync(FULL, v, o);
            v = mx ? fmaxf(v, y) : fminf(v, y);
        }
        if ((threadIdx.x & 31) == 0) {
            if (mx) atomicMax(&a[k], f2ord(v));
            else atomicMin(&a[k], f2ord(v));
        }
    }
}

// ------------------------------------------------------- large levels --
struct Task {
    int node, start, count, depth;
    float clo[3], chi[3];
};
struct Split {
    int axis, bin, nl, pad;
};
struct Chunk {
    int task, start, count, first;
};

// bins per task: [axis][bin] x {cnt, lo3, hi3} as ordered uints (the
// children's centroid bounds are gathered by k_count_left instead)
constexpr int BIN_WORDS = 7;
constexpr int PART_IPT = CHUNK / CHUNK_T;  // 8 consecutive positions per thread
__host__ __device__ __forceinline__ uint32_t bin_init(int w) {
    return w == 0 ? 0u : (w <= 3 ? 0xFFFFFFFFu : 0u);  // cnt 0, lo: min (from max), hi: max (from 0)
}
constexpr int TASK_BIN_WORDS = 3 * kBins * BIN_WORDS;

// The level loop runs ahead of the host: task and chunk counts stay on the
// device, grids are sized for upper bounds, and threads past the count exit
// (or write zeros where a scan covers the whole bound).
__global__ void k_chunk_counts(const Task* __restrict__ tasks, const int* __restrict__ d_T, int Tb,
                               int* __restrict__ cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < Tb) cnt[i] = i < *d_T ? (tasks[i].count + CHUNK - 1) / CHUNK : 0;
}

__global__ void k_fill_chunks(const Task* __restrict__ tasks, const int* __restrict__ d_T,
                              const int* __restrict__ off, Chunk* __restrict__ chunks) {
    const int t = blockIdx.x;
    if (t >= *d_T) return;
    const Task tk = tasks[t];
    const int nc = (tk.count + CHUNK - 1) / CHUNK;
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        Chunk ch;
        ch.task = t;
        ch.start = tk.start + c * CHUNK;
        ch.count = min(CHUNK, tk.count - c * CHUNK);
        ch.first = off[t];
        chunks[off[t] + c] = ch;
    }
}

__global__ void k_clear_bins(uint32_t* __restrict__ bins, const int* __restrict__ d_T) {
    const size_t total = (size_t)*d_T * TASK_BIN_WORDS;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        bins[i] = bin_init((int)(i % BIN_WORDS));
    }
}

__global__ void __launch_bounds__(CHUNK_T) k_bin_large(const Chunk* __restrict__ chunks, const Task* __restrict__ tasks,
                                                       const int* __restrict__ perm, const float4* __restrict__ plo,
                                                       const float4* __restrict__ phi, uint32_t* __restrict__ gbins,
                                                       const int* __restrict__ d_C) {
    __shared__ uint32_t sb[TASK_BIN_WORDS];
    if (blockIdx.x >= *d_C) return;
    const Chunk ch = chunks[blockIdx.x];
    const Task tk = tasks[ch.task];
    for (int i = threadIdx.x; i < TASK_BIN_WORDS; i += CHUNK_T) sb[i] = bin_init(i % BIN_WORDS);
    float k3[3];
#pragma unroll
    for (int a = 0; a < 3; a++) k3[a] = bin_scale(tk.clo[a], tk.chi[a]);
    __syncthreads();
    // PART_IPT consecutive positions per thread; a run of primitives in the
    // same bin of an axis (neighbours in a mesh usually are) is merged in
    // registers and reaches the shared bins as one set of atomics
    int rb[3] = {-1, -1, -1};
    uint32_t rc[3] = {0u, 0u, 0u};
    float rl[3][3], rh[3][3];
    auto flush = [&](int a) {
        uint32_t* w = sb + (a * kBins + rb[a]) * BIN_WORDS;
        atomicAdd(&w[0], rc[a]);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            atomicMin(&w[1 + k], f2ord(rl[a][k]));
            atomicMax(&w[4 + k], f2ord(rh[a][k]));
        }
    };
#pragma unroll
    for (int j = 0; j < PART_IPT; j++) {
        const int i = threadIdx.x * PART_IPT + j;
        if (i < ch.count) {
            const int p = perm[ch.start + i];
            const float4 l = plo[p], h = phi[p];
            const float L[3] = {l.x, l.y, l.z}, H[3] = {h.x, h.y, h.z};
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const int b = bin_of(centroid(L[a], H[a]), tk.clo[a], k3[a]);
                if (b != rb[a]) {
                    if (rb[a] >= 0) flush(a);
                    rb[a] = b;
                    rc[a] = 1u;
#pragma unroll
                    for (int k = 0; k < 3; k++) { rl[a][k] = L[k]; rh[a][k] = H[k]; }
                } else {
                    rc[a]++;
#pragma unroll
                    for (int k = 0; k < 3; k++) { rl[a][k] = fminf(rl[a][k], L[k]); rh[a][k] = fmaxf(rh[a][k], H[k]); }
                }
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
        if (rb[a] >= 0) flush(a);
    __syncthreads();
    uint32_t* g = gbins + (size_t)ch.task * TASK_BIN_WORDS;
    for (int i = threadIdx.x; i < TASK_BIN_WORDS; i += CHUNK_T) {
        const int w = i % BIN_WORDS;
        const uint32_t v = sb[i];
        if (w == 0) { if (v) atomicAdd(&g[i], v); }
        else if (w <= 3) { if (v != 0xFFFFFFFFu) atomicMin(&g[i], v); }
        else if (v) atomicMax(&g[i], v);
    }
}

struct BinBox {
    float lo[3], hi[3];
    int cnt;
};

__device__ __forceinline__ void box_merge(BinBox& a, const BinBox& b) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        a.lo[k] = fminf(a.lo[k], b.lo[k]);
        a.hi[k] = fmaxf(a.hi[k], b.hi[k]);
    }
    a.cnt += b.cnt;
}
__device__ __forceinline__ BinBox shfl_box(const BinBox& v, int src_delta, bool up) {
    BinBox r;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        r.lo[k] = up ? __shfl_up_sync(FULL, v.lo[k], src_delta) : __shfl_down_sync(FULL, v.lo[k], src_delta);
        r.hi[k] = up ? __shfl_up_sync(FULL, v.hi[k], src_delta) : __shfl_down_sync(FULL, v.hi[k], src_delta);
    }
    r.cnt = up ? __shfl_up_sync(FULL, v.cnt, src_delta) : __shfl_down_sync(FULL, v.cnt, src_delta);
    return r;
}

// Prefix (bins 0..lane) and suffix (bins lane..31) of one axis.
__device__ void prefix_suffix(const BinBox& mine, BinBox& pre, BinBox& suf) {
    const int lane = threadIdx.x & 31;
    pre = mine;
    suf = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        BinBox y = shfl_box(pre, o, true);
        if (lane >= o) box_merge(pre, y);
        BinBox z = shfl_box(suf, o, false);
        if (lane + o < 32) box_merge(suf, z);
    }
}

__device__ BinBox load_bin(const uint32_t* w) {
    BinBox b;
    b.cnt = (int)w[0];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        b.lo[k] = b.cnt ? ord2f(w[1 + k]) : FLT_MAX;
        b.hi[k] = b.cnt ? ord2f(w[4 + k]) : -FLT_MAX;
    }
    return b;
}

// One warp per task: best (axis, bin) by SAH; writes the split, the two
// child nodes (ids base + 2t, base + 2t + 1) and their task descriptors.
__global__ void k_split_large(const Task* __restrict__ tasks, const int* __restrict__ d_T,
                              const uint32_t* __restrict__ gbins, Split* __restrict__ splits, Task* __restrict__ kids,
                              uint32_t* __restrict__ kcb, Node2* __restrict__ nodes, const int* __restrict__ d_node_base,
                              int max_leaf, int max_sah_depth) {
    const int t = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (t >= *d_T) return;
    const int node_base = *d_node_base;
    const int lane = threadIdx.x & 31;
    const Task tk = tasks[t];
    const uint32_t* g = gbins + (size_t)t * TASK_BIN_WORDS;
    float best = FLT_MAX;
    int best_axis = -1, best_bin = -1;
    for (int a = 0; a < 3; a++) {
        BinBox mine = load_bin(g + (a * kBins + lane) * BIN_WORDS), pre, suf;
        prefix_suffix(mine, pre, suf);
        BinBox right = shfl_box(suf, 1, false);
        float cost = FLT_MAX;
        if (lane < kBins - 1 && pre.cnt > 0 && right.cnt > 0)
            cost = pre.cnt * half_area(pre.lo[0], pre.lo[1], pre.lo[2], pre.hi[0], pre.hi[1], pre.hi[2]) +
                   right.cnt * half_area(right.lo[0], right.lo[1], right.lo[2], right.hi[0], right.hi[1], right.hi[2]);
        // warp argmin, ties toward the lower bin
        float c = cost;
        int b = lane;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const float c2 = __shfl_xor_sync(FULL, c, o);
            const int b2 = __shfl_xor_sync(FULL, b, o);
            if (c2 < c || (c2 == c && b2 < b)) { c = c2; b = b2; }
        }
        if (c < best) { best = c; best_axis = a; best_bin = b; }
    }
    const bool median = best_axis < 0 || best == FLT_MAX || tk.depth >= max_sah_depth;
    BinBox L, R;
    int nl;
    const Node2 pn = nodes[tk.node];
    if (!median) {
        BinBox mine = load_bin(g + (best_axis * kBins + lane) * BIN_WORDS), pre, suf;
        prefix_suffix(mine, pre, suf);
        BinBox right = shfl_box(suf, 1, false);
        L = pre;
        R = right;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            L.lo[k] = __shfl_sync(FULL, pre.lo[k], best_bin); L.hi[k] = __shfl_sync(FULL, pre.hi[k], best_bin);
            R.lo[k] = __shfl_sync(FULL, right.lo[k], best_bin); R.hi[k] = __shfl_sync(FULL, right.hi[k], best_bin);
        }
        nl = __shfl_sync(FULL, pre.cnt, best_bin);
    } else {
        nl = tk.count / 2;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            L.lo[k] = R.lo[k] = pn.lo[k];
            L.hi[k] = R.hi[k] = pn.hi[k];
        }
    }
    if (lane == 0) {
        Split sp;
        sp.axis = median ? -1 : best_axis;
        sp.bin = best_bin;
        sp.nl = nl;
        sp.pad = 0;
        splits[t] = sp;
        const int lid = node_base + 2 * t, rid = lid + 1;
        nodes[tk.node].a = lid;
        nodes[tk.node].b = rid;
        const int cnt[2] = {nl, tk.count - nl};
        const int st[2] = {tk.start, tk.start + nl};
        for (int s = 0; s < 2; s++) {
            const BinBox& B = s ? R : L;
            Node2 nd;
            for (int k = 0; k < 3; k++) { nd.lo[k] = B.lo[k]; nd.hi[k] = B.hi[k]; }
            nd.a = 0;
            nd.b = 0;
            if (cnt[s] <= max_leaf) { nd.a = st[s]; nd.b = -cnt[s]; }
            nodes[lid + s] = nd;
            Task kt;
            kt.node = lid + s;
            kt.start = st[s];
            kt.count = cnt[s];
            kt.depth = tk.depth + 1;
            for (int k = 0; k < 3; k++) { kt.clo[k] = 0.f; kt.chi[k] = 0.f; }  // from kcb, after k_count_left
            kids[2 * t + s] = kt;
            for (int k = 0; k < 6; k++) kcb[(size_t)(2 * t + s) * 6 + k] = k < 3 ? 0xFFFFFFFFu : 0u;
        }
    }
}

__device__ __forceinline__ bool goes_left(const Task& tk, const Split& sp, int pos, const float4& l,
                                          const float4& h) {
    if (sp.axis < 0) return pos - tk.start < sp.nl;
    const float L = sp.axis == 0 ? l.x : (sp.axis == 1 ? l.y : l.z);
    const float H = sp.axis == 0 ? h.x : (sp.axis == 1 ? h.y : h.z);
    const float k = bin_scale(tk.clo[sp.axis], tk.chi[sp.axis]);
    return bin_of(centroid(L, H), tk.clo[sp.axis], k) <= sp.bin;
}


__global__ void __launch_bounds__(CHUNK_T) k_count_left(const Chunk* __restrict__ chunks, const Task* __restrict__ tasks,
                                                        const Split* __restrict__ splits, const int* __restrict__ perm,
                                                        const float4* __restrict__ plo, const float4* __restrict__ phi,
                                                        int* __restrict__ chunk_left, uint32_t* __restrict__ kcb,
                                                        const int* __restrict__ d_C, uint8_t* __restrict__ side) {
    __shared__ int ws[CHUNK_T / 32];
    if (blockIdx.x >= *d_C) return;  // (the scan over the bound reads stale counts only after the last chunk)
    const Chunk ch = chunks[blockIdx.x];
    const Task tk = tasks[ch.task];
    const Split sp = splits[ch.task];
    int c = 0;
    // centroid bounds of each side: [side][min xyz, max xyz]
    float cb[2][6];
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int k = 0; k < 3; k++) { cb[s][k] = FLT_MAX; cb[s][3 + k] = -FLT_MAX; }
#pragma unroll
    for (int j = 0; j < PART_IPT; j++) {
        const int i = threadIdx.x * PART_IPT + j;
        if (i < ch.count) {
            const int p = perm[ch.start + i];
            const float4 l = plo[p], h = phi[p];
            const bool left = goes_left(tk, sp, ch.start + i, l, h);
            side[ch.start + i] = left;  // k_scatter reads this instead of the boxes
            c += left;
            const float C[3] = {centroid(l.x, h.x), centroid(l.y, h.y), centroid(l.z, h.z)};
#pragma unroll
            for (int k = 0; k < 3; k++) {
                cb[0][k] = left ? fminf(cb[0][k], C[k]) : cb[0][k];
                cb[0][3 + k] = left ? fmaxf(cb[0][3 + k], C[k]) : cb[0][3 + k];
                cb[1][k] = left ? cb[1][k] : fminf(cb[1][k], C[k]);
                cb[1][3 + k] = left ? cb[1][3 + k] : fmaxf(cb[1][3 + k], C[k]);
            }
        }
    }
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int k = 0; k < 6; k++) {
            float v = cb[s][k];
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const float y = __shfl_xor_sync(FULL, v, o);
                v = k < 3 ? fminf(v, y) : fmaxf(v, y);
            }
            cb[s][k] = v;
        }
    if ((threadIdx.x & 31) < 2) {  // lane s: side s, when the warp saw any of it
        const int s = threadIdx.x & 31;
        const float* v = s ? cb[1] : cb[0];
        if (v[0] <= v[3]) {
            uint32_t* dst = kcb + (size_t)(2 * ch.task + s) * 6;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                atomicMin(&dst[k], f2ord(v[k]));
                atomicMax(&dst[3 + k], f2ord(v[3 + k]));
            }
        }
    }
    int total;
    block_exclusive_scan<CHUNK_T>(c, ws, total);
    if (threadIdx.x == 0) chunk_left[blockIdx.x] = total;
}

__global__ void __launch_bounds__(CHUNK_T) k_scatter(const Chunk* __restrict__ chunks, const Task* __restrict__ tasks,
                                                     const Split* __restrict__ splits, const int* __restrict__ perm,
                                                     const uint8_t* __restrict__ side, const int* __restrict__ left_off,
                                                     int* __restrict__ out, const int* __restrict__ d_C) {
    __shared__ int ws[CHUNK_T / 32];
    if (blockIdx.x >= *d_C) return;
    const Chunk ch = chunks[blockIdx.x];
    const Task tk = tasks[ch.task];
    const Split sp = splits[ch.task];
    bool f[PART_IPT];
    int pv[PART_IPT];
    int c = 0;
    for (int k = 0; k < PART_IPT; k++) {
        const int i = threadIdx.x * PART_IPT + k;
        f[k] = false;
        pv[k] = -1;
        if (i < ch.count) {
            pv[k] = perm[ch.start + i];
            f[k] = side[ch.start + i] != 0;
            c += f[k];
        }
    }
    int total;
    int lr = block_exclusive_scan<CHUNK_T>(c, ws, total);  // lefts before my first element
    const int left_before = left_off[blockIdx.x] - left_off[ch.first];
    const int right_before = (ch.start - tk.start) - left_before;
    for (int k = 0; k < PART_IPT; k++) {
        const int i = threadIdx.x * PART_IPT + k;
        if (i < ch.count) {
            const int dst = f[k] ? tk.start + left_before + lr : tk.start + sp.nl + right_before + (i - lr);
            lr += f[k];
            out[dst] = pv[k];
        }
    }
}

__global__ void k_copy_back(const Chunk* __restrict__ chunks, const int* __restrict__ src, int* __restrict__ dst,
                            const int* __restrict__ d_C) {
    if (blockIdx.x >= *d_C) return;
    const Chunk ch = chunks[blockIdx.x];
    for (int i = threadIdx.x; i < ch.count; i += blockDim.x) dst[ch.start + i] = src[ch.start + i];
}

__global__ void k_classify_flags(const Task* __restrict__ kids, const int* __restrict__ d_T, int Kb, int max_leaf,
                                 int small_task, int* __restrict__ is_large, int* __restrict__ is_small) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Kb) return;
    if (i >= 2 * *d_T) {  // past this level's kids: zeros for the scans over the bound
        is_large[i] = 0;
        is_small[i] = 0;
        return;
    }
    const int c = kids[i].count;
    is_large[i] = c > small_task;
    is_small[i] = c > max_leaf && c <= small_task;
}

__global__ void k_compact_kids(const Task* __restrict__ kids, const int* __restrict__ d_T,
                               const int* __restrict__ is_large, const int* __restrict__ large_off,
                               const int* __restrict__ is_small, const int* __restrict__ small_off,
                               Task* __restrict__ next, int max_large, Task* __restrict__ small, int max_small,
                               const int* __restrict__ small_base, const uint32_t* __restrict__ kcb,
                               int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * *d_T) return;
    Task t = kids[i];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        t.clo[k] = ord2f(kcb[(size_t)i * 6 + k]);
        t.chi[k] = ord2f(kcb[(size_t)i * 6 + 3 + k]);
    }
    if (is_large[i]) {
        if (large_off[i] < max_large) next[large_off[i]] = t;
        else atomicOr(status, 8);
    }
    if (is_small[i]) {
        const int at = *small_base + small_off[i];
        if (at < max_small) small[at] = t;
        else atomicOr(status, 8);
    }
}

// End of a level: node ids advance past this level's kids, the small list
// grows, the next level's task count becomes current and is logged for the
// host (which reads it one level behind).
__global__ void k_level_end(int* __restrict__ d_T, int* __restrict__ d_node_count, int* __restrict__ small_base,
                            const int* __restrict__ tot, int max_large, int max_small, int* __restrict__ log_T,
                            int* __restrict__ status) {
    *d_node_count += 2 * *d_T;
    *small_base = min(*small_base + tot[1], max_small);
    const int tn = tot[0];
    if (tn > max_large) atomicOr(status, 8);
    *d_T = min(tn, max_large);
    *log_T = *d_T;
}

// ----------------------------------------------------------- small tasks --
// One CTA finishes the subtree of a task of <= small_task primitives in
// shared memory.  Node ids come from the task's reserved range, handed out
// in the CTA's fixed processing order (deterministic).
struct SubTask {
    int node, lstart, count, depth;
};

// A subtree of at most WARP_TASK primitives handed from k_build_small to
// k_build_warp: its node (already written by its parent), its range in the
// permutation, and the first of the 2 * count - 2 node ids reserved for it.
constexpr int WARP_TASK = 32;
struct WTask {
    int node, start, count_depth, nbase;  // count_depth: count | depth << 8
};

__global__ void k_reserve(const Task* __restrict__ small, int S, int* __restrict__ need) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < S) need[i] = 2 * small[i].count - 2;
}

template <int T>
__device__ void block_minmax6(float (&v)[6], float* sh) {
    // v[0..2] min-reduced, v[3..5] max-reduced over the block; result in all threads
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; k++) {
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const float y = __shfl_xor_sync(FULL, v[k], o);
            v[k] = k < 3 ? fminf(v[k], y) : fmaxf(v[k], y);
        }
    }
    __syncthreads();
    if (lane == 0)
        for (int k = 0; k < 6; k++) sh[w * 6 + k] = v[k];
    __syncthreads();
    for (int k = 0; k < 6; k++) {
        float r = sh[k];
        for (int j = 1; j < T / 32; j++) r = k < 3 ? fminf(r, sh[j * 6 + k]) : fmaxf(r, sh[j * 6 + k]);
        v[k] = r;
    }
    __syncthreads();
}

__device__ __forceinline__ void build_small_task(int task, const Task* __restrict__ small,
                                                 const int* __restrict__ res_off, int res_base, int* __restrict__ perm,
                                                 const float4* __restrict__ plo, const float4* __restrict__ phi,
                                                 Node2* __restrict__ nodes, int max_leaf, int max_sah_depth,
                                                 int small_task, int warp_task, WTask* __restrict__ wq, int wq_cap,
                                                 int* __restrict__ wq_count, int* __restrict__ status) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    const Task tk = small[task];
    const int n = tk.count;
    float* blo = sm;                                  // [3][small_task]
    float* bhi = blo + 3 * small_task;                // [3][small_task]
    int* gidx = reinterpret_cast<int*>(bhi + 3 * small_task);  // [small_task]
    unsigned short* pa = reinterpret_cast<unsigned short*>(gidx + small_task);
    unsigned short* pb = pa + small_task;
    uint32_t* bins = reinterpret_cast<uint32_t*>(pb + small_task + (small_task & 1));  // [3][32][7]
    __shared__ SubTask stack[SMALL_STACK];
    __shared__ int sp_top, next_node, s_axis, s_bin, s_done;
    __shared__ SubTask cur;
    __shared__ float red[6 * (SMALL_T / 32)];
    __shared__ float s_cost[3];
    __shared__ int s_cbin[3];
    __shared__ float s_cbox[3][12];  // per axis: left box, right box of its best split
    __shared__ int ws[SMALL_T / 32];

    for (int i = threadIdx.x; i < n; i += SMALL_T) {
        const int p = perm[tk.start + i];
        gidx[i] = p;
        const float4 l = plo[p], h = phi[p];
        blo[i] = l.x; blo[small_task + i] = l.y; blo[2 * small_task + i] = l.z;
        bhi[i] = h.x; bhi[small_task + i] = h.y; bhi[2 * small_task + i] = h.z;
        pa[i] = (unsigned short)i;
    }
    if (threadIdx.x == 0) {
        sp_top = 1;
        SubTask r;
        r.node = tk.node; r.lstart = 0; r.count = n; r.depth = tk.depth;
        stack[0] = r;
        next_node = res_base + res_off[task];
    }
    __syncthreads();
    while (true) {
        if (threadIdx.x == 0) {
            s_done = sp_top == 0;
            if (!s_done) cur = stack[--sp_top];
        }
        __syncthreads();
        if (s_done) break;
        const SubTask st = cur;
        if (st.count <= max_leaf) {
            if (threadIdx.x == 0) {
                nodes[st.node].a = tk.start + st.lstart;
                nodes[st.node].b = -st.count;
            }
            __syncthreads();
            continue;
        }
        if (st.count <= warp_task) {  // the rest of this subtree goes to one warp (k_build_warp)
            if (threadIdx.x == 0) {
                const int slot = atomicAdd(wq_count, 1);
                if (slot < wq_cap) {
                    WTask w;
                    w.node = st.node;
                    w.start = tk.start + st.lstart;
                    w.count_depth = st.count | (st.depth << 8);
                    w.nbase = next_node;
                    wq[slot] = w;
                } else {
                    atomicOr(status, 2);
                }
                next_node += 2 * st.count - 2;
            }
            __syncthreads();
            continue;
        }
        // centroid bounds of this range
        float cb[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = threadIdx.x; i < st.count; i += SMALL_T) {
            const int q = pa[st.lstart + i];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const float c = centroid(blo[a * small_task + q], bhi[a * small_task + q]);
                cb[a] = fminf(cb[a], c);
                cb[3 + a] = fmaxf(cb[3 + a], c);
            }
        }
        block_minmax6<SMALL_T>(cb, red);
        float k3[3];
#pragma unroll
        for (int a = 0; a < 3; a++) k3[a] = bin_scale(cb[a], cb[3 + a]);
        for (int i = threadIdx.x; i < 3 * kBins * BIN_WORDS; i += SMALL_T) bins[i] = bin_init(i % BIN_WORDS);
        __syncthreads();
        // each thread bins `per` consecutive positions; runs in one bin of an
        // axis are merged in registers first (as in k_bin_large)
        const int per = (st.count + SMALL_T - 1) / SMALL_T;  // <= small_task / SMALL_T
        const int i0 = threadIdx.x * per, i1 = min(i0 + per, st.count);
        {
            int rb[3] = {-1, -1, -1};
            uint32_t rc[3] = {0u, 0u, 0u};
            float rl[3][3], rh[3][3];
            auto flush = [&](int a) {
                uint32_t* w = bins + (a * kBins + rb[a]) * BIN_WORDS;
                atomicAdd(&w[0], rc[a]);
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    atomicMin(&w[1 + k], f2ord(rl[a][k]));
                    atomicMax(&w[4 + k], f2ord(rh[a][k]));
                }
            };
            for (int i = i0; i < i1; i++) {
                const int q = pa[st.lstart + i];
                float L[3], H[3];
#pragma unroll
                for (int a = 0; a < 3; a++) { L[a] = blo[a * small_task + q]; H[a] = bhi[a * small_task + q]; }
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const int b = bin_of(centroid(L[a], H[a]), cb[a], k3[a]);
                    if (b != rb[a]) {
                        if (rb[a] >= 0) flush(a);
                        rb[a] = b;
                        rc[a] = 1u;
#pragma unroll
                        for (int k = 0; k < 3; k++) { rl[a][k] = L[k]; rh[a][k] = H[k]; }
                    } else {
                        rc[a]++;
#pragma unroll
                        for (int k = 0; k < 3; k++) { rl[a][k] = fminf(rl[a][k], L[k]); rh[a][k] = fmaxf(rh[a][k], H[k]); }
                    }
                }
            }
#pragma unroll
            for (int a = 0; a < 3; a++)
                if (rb[a] >= 0) flush(a);
        }
        __syncthreads();
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (warp < 3) {
            const uint32_t* w = bins + (warp * kBins + lane) * BIN_WORDS;
            BinBox mine = load_bin(w), pre, suf;
            prefix_suffix(mine, pre, suf);
            BinBox right = shfl_box(suf, 1, false);
            float cost = FLT_MAX;
            if (lane < kBins - 1 && pre.cnt > 0 && right.cnt > 0)
                cost = pre.cnt * half_area(pre.lo[0], pre.lo[1], pre.lo[2], pre.hi[0], pre.hi[1], pre.hi[2]) +
                       right.cnt * half_area(right.lo[0], right.lo[1], right.lo[2], right.hi[0], right.hi[1], right.hi[2]);
            float c = cost;
            int b = lane;
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const float c2 = __shfl_xor_sync(FULL, c, o);
                const int b2 = __shfl_xor_sync(FULL, b, o);
                if (c2 < c || (c2 == c && b2 < b)) { c = c2; b = b2; }
            }
            // the children's boxes: the bins' union on each side of the split
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const float l0 = __shfl_sync(FULL, pre.lo[k], b), l1 = __shfl_sync(FULL, pre.hi[k], b);
                const float r0 = __shfl_sync(FULL, right.lo[k], b), r1 = __shfl_sync(FULL, right.hi[k], b);
                if (lane == 0) {
                    s_cbox[warp][k] = l0; s_cbox[warp][3 + k] = l1;
                    s_cbox[warp][6 + k] = r0; s_cbox[warp][9 + k] = r1;
                }
            }
            if (lane == 0) { s_cost[warp] = c; s_cbin[warp] = b; }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            float best = FLT_MAX;
            int ba = -1, bb = -1;
            for (int a = 0; a < 3; a++)
                if (s_cost[a] < best) { best = s_cost[a]; ba = a; bb = s_cbin[a]; }
            if (ba < 0 || st.depth >= max_sah_depth) { ba = -1; bb = -1; }
            s_axis = ba;
            s_bin = bb;
        }
        __syncthreads();
        const int axis = s_axis, sbin = s_bin;
        // stable partition of pa[lstart, lstart+count) in one scan: each
        // thread flags its consecutive positions, counts its lefts, and
        // writes lefts after the lefts before it and rights after all lefts
        uint32_t fl = 0u;
        int mine_l = 0;
        for (int i = i0; i < i1; i++) {
            const int q = pa[st.lstart + i];
            const bool f = axis < 0 ? i < st.count / 2
                                    : bin_of(centroid(blo[axis * small_task + q], bhi[axis * small_task + q]), cb[axis],
                                             k3[axis]) <= sbin;
            fl |= (f ? 1u : 0u) << (i - i0);
            mine_l += f;
        }
        int nl;
        int lb = block_exclusive_scan<SMALL_T>(mine_l, ws, nl);
        int rb_ = (i0 - lb);  // rights before my first position
        for (int i = i0; i < i1; i++) {
            const unsigned short q = pa[st.lstart + i];
            if ((fl >> (i - i0)) & 1u) pb[st.lstart + lb++] = q;
            else pb[st.lstart + nl + rb_++] = q;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < st.count; i += SMALL_T) pa[st.lstart + i] = pb[st.lstart + i];
        __syncthreads();
        // child boxes: from the bins, or by reduction after a median split
        float bl[6], br[6];
        if (axis >= 0) {
#pragma unroll
            for (int k = 0; k < 6; k++) { bl[k] = s_cbox[axis][k]; br[k] = s_cbox[axis][6 + k]; }
        } else {
#pragma unroll
            for (int k = 0; k < 3; k++) { bl[k] = br[k] = FLT_MAX; bl[3 + k] = br[3 + k] = -FLT_MAX; }
            for (int i = threadIdx.x; i < st.count; i += SMALL_T) {
                const int q = pa[st.lstart + i];
                float* B = i < nl ? bl : br;
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    B[a] = fminf(B[a], blo[a * small_task + q]);
                    B[3 + a] = fmaxf(B[3 + a], bhi[a * small_task + q]);
                }
            }
            block_minmax6<SMALL_T>(bl, red);
            block_minmax6<SMALL_T>(br, red);
        }
        if (threadIdx.x == 0) {
            const int lid = next_node, rid = next_node + 1;
            next_node += 2;
            nodes[st.node].a = lid;
            nodes[st.node].b = rid;
            Node2 L, R;
            for (int a = 0; a < 3; a++) {
                L.lo[a] = bl[a]; L.hi[a] = bl[3 + a];
                R.lo[a] = br[a]; R.hi[a] = br[3 + a];
            }
            L.a = tk.start + st.lstart; L.b = -nl;
            R.a = tk.start + st.lstart + nl; R.b = -(st.count - nl);
            if (nl > max_leaf) L.b = 0;
            if (st.count - nl > max_leaf) R.b = 0;
            nodes[lid] = L;
            nodes[rid] = R;
            if (sp_top + 2 > SMALL_STACK) {
                atomicOr(status, 1);  // cannot happen with the depth bound; reported, never silent
            } else {
                SubTask sr, sl;
                sr.node = rid; sr.lstart = st.lstart + nl; sr.count = st.count - nl; sr.depth = st.depth + 1;
                sl.node = lid; sl.lstart = st.lstart; sl.count = nl; sl.depth = st.depth + 1;
                if (sr.count > max_leaf) stack[sp_top++] = sr;
                if (sl.count > max_leaf) stack[sp_top++] = sl;
            }
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += SMALL_T) perm[tk.start + i] = gidx[pa[i]];
}

// One CTA per small task.
__global__ void __launch_bounds__(SMALL_T) k_build_small(const Task* __restrict__ small, const int* __restrict__ res_off,
                                                         int res_base, int* __restrict__ perm,
                                                         const float4* __restrict__ plo, const float4* __restrict__ phi,
                                                         Node2* __restrict__ nodes, int max_leaf, int max_sah_depth,
                                                         int small_task, int warp_task, WTask* __restrict__ wq,
                                                         int wq_cap, int* __restrict__ wq_count,
                                                         int* __restrict__ status) {
    build_small_task(blockIdx.x, small, res_off, res_base, perm, plo, phi, nodes, max_leaf, max_sah_depth, small_task,
                     warp_task, wq, wq_cap, wq_count, status);
}

// Persistent CTAs take small tasks from a work counter until the device's
// task count (*d_S) is reached; the node ids still come from each task's
// reserved range, so the tree does not depend on which CTA took a task.
__global__ void __launch_bounds__(SMALL_T) k_build_small_loop(const Task* __restrict__ small, const int* __restrict__ d_S,
                                                              int* __restrict__ work, const int* __restrict__ res_off,
                                                              const int* __restrict__ d_res_base, int* __restrict__ perm,
                                                              const float4* __restrict__ plo,
                                                              const float4* __restrict__ phi,
                                                              Node2* __restrict__ nodes, int max_leaf,
                                                              int max_sah_depth, int small_task, int warp_task,
                                                              WTask* __restrict__ wq, int wq_cap,
                                                              int* __restrict__ wq_count, int* __restrict__ status) {
    __shared__ int s_task;
    const int S = *d_S, res_base = *d_res_base;
    for (;;) {
        __syncthreads();  // the previous task is done with shared memory
        if (threadIdx.x == 0) s_task = atomicAdd(work, 1);
        __syncthreads();
        const int t = s_task;
        if (t >= S) break;
        build_small_task(t, small, res_off, res_base, perm, plo, phi, nodes, max_leaf, max_sah_depth, small_task,
                         warp_task, wq, wq_cap, wq_count, status);
    }
}

// One warp finishes a subtree of at most 32 primitives with an exact SAH
// sweep (every split between consecutive centroids along each axis, cost
// N_L*A(L) + N_R*A(R) as above).  The primitives are sorted by centroid
// along each axis once, by a bitonic network over the lanes (ties by
// primitive slot); a split partitions all three orders stably, so every
// node's primitives stay a contiguous, still sorted range of each order.
// The nodes of one depth own disjoint ranges, so a whole level is split in
// one pass: lane l works on position l, and prefix/suffix scans, the
// cheapest-split search (ties: lower split, then lower axis) and the
// partition are segmented by node range.  Node ids are handed out from the
// reserved range level by level, in position order, so the tree is
// deterministic.
constexpr int WB_T = 128;  // 4 warps per CTA, one subtree each at a time
constexpr int WB_W = WB_T / 32;

__device__ __forceinline__ float box_half_area(const float (&b)[6]) {
    return half_area(b[0], b[1], b[2], b[3], b[4], b[5]);
}

__global__ void __launch_bounds__(WB_T) k_build_warp(const WTask* __restrict__ wq, const int* __restrict__ wq_count,
                                                     int wq_cap, int* __restrict__ perm,
                                                     const float4* __restrict__ plo, const float4* __restrict__ phi,
                                                     Node2* __restrict__ nodes, int max_leaf, int max_sah_depth) {
    __shared__ float s_box[WB_W][6][32];          // lo xyz, hi xyz per slot
    __shared__ int s_idx[WB_W][32];               // primitive per slot
    __shared__ unsigned char s_ord[WB_W][3][32];  // per axis: position -> slot
    __shared__ unsigned char s_side[WB_W][32];    // per slot: 1 = left of its node's split
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int total = min(*wq_count, wq_cap);
    for (int t = blockIdx.x * WB_W + w; t < total; t += gridDim.x * WB_W) {
        const WTask wt = wq[t];
        const int cnt = wt.count_depth & 255;
        // load this subtree's primitives, one per lane
        float b[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (lane < cnt) {
            const int p = perm[wt.start + lane];
            const float4 l = plo[p], h = phi[p];
            b[0] = l.x; b[1] = l.y; b[2] = l.z;
            b[3] = h.x; b[4] = h.y; b[5] = h.z;
            s_idx[w][lane] = p;
#pragma unroll
            for (int k = 0; k < 6; k++) s_box[w][k][lane] = b[k];
        }
        // one bitonic sort per axis: (centroid key, slot), idle lanes last
#pragma unroll
        for (int a = 0; a < 3; a++) {
            uint32_t key = lane < cnt ? f2ord(centroid(b[a], b[3 + a])) : 0xFFFFFFFFu;
            int val = lane;
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const uint32_t ok = __shfl_xor_sync(FULL, key, j);
                    const int ov = __shfl_xor_sync(FULL, val, j);
                    const bool less = ok < key || (ok == key && ov < val);
                    const bool take = (((lane & j) == 0) == ((lane & k) == 0)) ? less : !less;
                    if (take) { key = ok; val = ov; }
                }
            }
            s_ord[w][a][lane] = (unsigned char)val;
        }
        __syncwarp();
        // this lane's node: range [s0, s1), id, depth; lanes past cnt own nothing
        int s0 = lane < cnt ? 0 : lane, s1 = lane < cnt ? cnt : lane + 1;
        int node = wt.node, depth = wt.count_depth >> 8;
        bool active = lane < cnt && cnt > max_leaf;
        int next = wt.nbase;
        while (__any_sync(FULL, active)) {
            const int len = s1 - s0;
            const int maxlen = __reduce_max_sync(FULL, active ? len : 0);
            const bool median = depth >= max_sah_depth;
            const unsigned seg_ge = ~((1u << s0) - 1u);  // lanes >= s0
            float best = INFINITY;
            int br = s0 + len / 2 - 1, ba = 0;
            float bl[6], bR[6];
#pragma unroll 1
            for (int a = 0; a < 3; a++) {
                float pre[6], suf[6];
                if (lane < cnt) {
                    const int s = s_ord[w][a][lane];
#pragma unroll
                    for (int k = 0; k < 6; k++) pre[k] = s_box[w][k][s];
                } else {
#pragma unroll
                    for (int k = 0; k < 3; k++) { pre[k] = FLT_MAX; pre[3 + k] = -FLT_MAX; }
                }
#pragma unroll
                for (int k = 0; k < 6; k++) suf[k] = pre[k];
                // segmented inclusive scans over each node's range
                for (int o = 1; o < maxlen; o <<= 1) {
                    const bool up = lane - o >= s0, dn = lane + o < s1;
#pragma unroll
                    for (int k = 0; k < 6; k++) {
                        const float x = __shfl_up_sync(FULL, pre[k], o);
                        const float y = __shfl_down_sync(FULL, suf[k], o);
                        if (up) pre[k] = k < 3 ? fminf(pre[k], x) : fmaxf(pre[k], x);
                        if (dn) suf[k] = k < 3 ? fminf(suf[k], y) : fmaxf(suf[k], y);
                    }
                }
                float right[6];
#pragma unroll
                for (int k = 0; k < 6; k++) right[k] = __shfl_down_sync(FULL, suf[k], 1);
                // positions without a right side, idle nodes and NaN costs read
                // +inf; ties go to the lower position, so a real split is chosen
                float cost = INFINITY;
                if (active && lane < s1 - 1 && !(median && a > 0)) {
                    cost = (float)(lane - s0 + 1) * box_half_area(pre) + (float)(s1 - lane - 1) * box_half_area(right);
                    if (!(cost <= FLT_MAX)) cost = INFINITY;
                }
                int r = lane;
                for (int o = 1; o < maxlen; o <<= 1) {  // segmented suffix minimum: the node's first lane ends with it
                    const float c2 = __shfl_down_sync(FULL, cost, o);
                    const int r2 = __shfl_down_sync(FULL, r, o);
                    if (lane + o < s1 && (c2 < cost || (c2 == cost && r2 < r))) { cost = c2; r = r2; }
                }
                cost = __shfl_sync(FULL, cost, s0);
                r = __shfl_sync(FULL, r, s0);
                if (median) r = s0 + len / 2 - 1;
                const bool take = active && (a == 0 || cost < best);
                if (take) {
                    best = cost;
                    br = r;
                    ba = a;
                }
                // each lane reads its own node's split lane
                const int src = take ? r : lane;
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    const float x = __shfl_sync(FULL, pre[k], src);
                    const float y = __shfl_sync(FULL, right[k], src);
                    if (take) { bl[k] = x; bR[k] = y; }
                }
            }
            const int nl = br - s0 + 1, nr = len - nl;
            // stable, segmented partition of the three orders: the first nl
            // positions of the winning axis' order go left
            if (active) s_side[w][s_ord[w][ba][lane]] = lane <= br;
            __syncwarp();
#pragma unroll
            for (int a = 0; a < 3; a++) {
                int s = 0;
                bool left = false;
                if (active) {
                    s = s_ord[w][a][lane];
                    left = s_side[w][s];
                }
                const unsigned bal = __ballot_sync(FULL, left);
                const int below = __popc(bal & lt & seg_ge);
                const int pos = left ? s0 + below : s0 + nl + (lane - s0 - below);
                __syncwarp();
                if (active) s_ord[w][a][pos] = (unsigned char)s;
            }
            __syncwarp();
            // two node ids per split node, in position order
            const bool lead = active && lane == s0;
            const unsigned leads = __ballot_sync(FULL, lead);
            const int mine = next + 2 * __popc(leads & lt);
            next += 2 * __popc(leads);
            const int lid = __shfl_sync(FULL, mine, s0);
            if (lead) {
                nodes[node].a = lid;
                nodes[node].b = lid + 1;
                Node2 L, R;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    L.lo[k] = bl[k]; L.hi[k] = bl[3 + k];
                    R.lo[k] = bR[k]; R.hi[k] = bR[3 + k];
                }
                L.a = wt.start + s0; L.b = nl > max_leaf ? 0 : -nl;
                R.a = wt.start + s0 + nl; R.b = nr > max_leaf ? 0 : -nr;
                nodes[lid] = L;
                nodes[lid + 1] = R;
            }
            if (active) {
                if (lane < s0 + nl) {
                    s1 = s0 + nl;
                    node = lid;
                    active = nl > max_leaf;
                } else {
                    s0 = s0 + nl;
                    node = lid + 1;
                    active = nr > max_leaf;
                }
                depth++;
            }
        }
        // leaf order = the axis-0 order (every leaf's range holds its primitives)
        if (lane < cnt) perm[wt.start + lane] = s_idx[w][s_ord[w][0][lane]];
        __syncwarp();
    }
}

__global__ void k_iota(int* __restrict__ p, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = i;
}

// ------------------------------------------------------ host-side build --
// Per host thread: pinned slots the level loop copies each level's task
// count into, and an event per level to wait on (created once per thread).
constexpr int kMaxLevels = 160;  // SAH depth 48, then median splits: far fewer levels
struct LevelLog {
    int* count = nullptr;
    cudaEvent_t ev[kMaxLevels] = {};
    bool ok = false;
    LevelLog() {
        if (cudaHostAlloc(reinterpret_cast<void**>(&count), sizeof(int) * kMaxLevels, cudaHostAllocDefault) !=
            cudaSuccess) {
            cudaGetLastError();
            return;
        }
        for (int i = 0; i < kMaxLevels; i++)
            if (cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                return;
            }
        ok = true;
    }
    ~LevelLog() {
        for (int i = 0; i < kMaxLevels; i++)
            if (ev[i]) cudaEventDestroy(ev[i]);
        if (count) cudaFreeHost(count);
    }
};
static LevelLog* level_log() {
    // one per device: events belong to the device that was current at creation
    constexpr int kDevices = 16;
    static thread_local std::unique_ptr<LevelLog> lg[kDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevices) {
        cudaGetLastError();
        set_error("build: no usable device for the level log");
        return nullptr;
    }
    if (!lg[dev]) lg[dev].reset(new (std::nothrow) LevelLog());
    if (!lg[dev] || !lg[dev]->ok) {
        set_error("build: pinned level log unavailable");
        return nullptr;
    }
    return lg[dev].get();
}

BuildConfig default_build_config() {
    BuildConfig c;
    if (const char* e = getenv("RTB200_MAX_LEAF")) c.max_leaf = std::max(1, std::min(4, atoi(e)));
    if (const char* e = getenv("RTB200_WARP_TASK")) c.warp_task = std::max(0, std::min(WARP_TASK, atoi(e)));
    if (const char* e = getenv("RTB200_SMALL_TASK")) c.small_task = std::max(WARP_TASK, std::min(32 * SMALL_T, atoi(e)));
    return c;
}

bool build_bvh2(const float4* d_lo, const float4* d_hi, int n, const BuildConfig& cfg, Bvh2Device& out,
                cudaStream_t s, const std::vector<int>* segments) {
    if (n <= 0) {
        set_error("build: empty input");
        return false;
    }
    if (cfg.max_leaf < 1 || cfg.max_leaf > 4) {
        set_error("build: max_leaf must be 1..4");
        return false;
    }
    if (cfg.small_task < WARP_TASK || cfg.small_task > 32 * SMALL_T) {  // k_build_small: <= 32 positions per thread
        set_error("build: small_task must be %d..%d", WARP_TASK, 32 * SMALL_T);
        return false;
    }
    std::vector<int> seg = segments ? *segments : std::vector<int>{0, n};
    const int S = (int)seg.size() - 1;
    if (S < 1 || seg.front() != 0 || seg.back() != n) {
        set_error("build: bad segment table");
        return false;
    }
    if (S > kMaxSegments) {
        set_error("build: %d scenes, at most %d per build", S, kMaxSegments);
        return false;
    }
    for (int i = 0; i < S; i++)
        if (seg[i + 1] <= seg[i]) {
            set_error("build: segment %d is empty", i);
            return false;
        }
    out.num_prims = n;
    out.num_roots = S;
    if (cfg.transient ? (!out.nodes.alloc_on((size_t)2 * n + 2, s) || !out.perm.alloc_on(n, s))
                      : (!out.nodes.alloc((size_t)2 * n + 2) || !out.perm.alloc(n)))
        return false;
    cudaMemsetAsync(out.nodes.p, 0, out.nodes.bytes(), s);
    int* perm = out.perm.p;
    // temporaries
    const int maxT = n / (cfg.small_task + 1) + 2;  // large tasks per level
    TmpBuf<int> tmp, dseg;
    TmpBuf<uint32_t> acc;
    TmpBuf<Task> tasks_a, tasks_b, kids, small;
    TmpBuf<Split> splits;
    TmpBuf<uint32_t> gbins;
    TmpBuf<int> flags, status;
    TmpBuf<uint32_t> kcb;  // per kid: centroid min xyz, max xyz (ordered)
    TmpBuf<uint8_t> side;  // per position: 1 = goes left at this level (k_count_left -> k_scatter)
    const int maxChunks = n / CHUNK + maxT + 2;
    TmpBuf<Chunk> chunks;
    TmpBuf<int> ccount, coff, cleft, cleftoff;
    const int maxSmall = n / (cfg.max_leaf + 1) + 2;
    if (!tmp.alloc(n, s) || !acc.alloc((size_t)12 * S, s) || !dseg.alloc(S + 1, s) || !tasks_a.alloc(maxT, s) ||
        !tasks_b.alloc(maxT, s) || !kids.alloc(2 * maxT, s) || !small.alloc(maxSmall, s) ||
        !splits.alloc(maxT, s) || !gbins.alloc((size_t)maxT * TASK_BIN_WORDS, s) ||
        !flags.alloc(4 * 2 * maxT + 8, s) || !chunks.alloc(maxChunks, s) || !ccount.alloc(maxT, s) ||
        !coff.alloc(maxT, s) || !cleft.alloc(maxChunks, s) || !cleftoff.alloc(maxChunks, s) || !status.alloc(1, s) ||
        !kcb.alloc((size_t)12 * maxT, s) || !side.alloc(n, s))
        return false;
    cudaMemsetAsync(status.p, 0, sizeof(int), s);
    k_iota<<<(n + 255) / 256, 256, 0, s>>>(perm, n);
    // per-segment root bounds, then the initial task lists (on the host, in
    // segment order, so node ids and task order are deterministic)
    std::vector<uint32_t> hacc((size_t)12 * S);
    for (int i = 0; i < S; i++)
        for (int k = 0; k < 12; k++) hacc[(size_t)i * 12 + k] = ((k >= 3 && k < 6) || k >= 9) ? 0u : 0xFFFFFFFFu;
    int maxcnt = 0;
    for (int i = 0; i < S; i++) maxcnt = std::max(maxcnt, seg[i + 1] - seg[i]);
    if (!RT_CUDA(cudaMemcpyAsync(acc.p, hacc.data(), hacc.size() * 4, cudaMemcpyHostToDevice, s)) ||
        !RT_CUDA(cudaMemcpyAsync(dseg.p, seg.data(), seg.size() * 4, cudaMemcpyHostToDevice, s)))
        return false;
    k_seg_bounds<<<dim3(std::min((maxcnt + 2047) / 2048, 64), S), 256, 0, s>>>(d_lo, d_hi, dseg.p, acc.p);
    if (!RT_CUDA(cudaMemcpyAsync(hacc.data(), acc.p, hacc.size() * 4, cudaMemcpyDeviceToHost, s)) ||
        !RT_CUDA(cudaStreamSynchronize(s)))
        return false;
    auto ordf = [](uint32_t u) {
        const uint32_t v = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
        float f;
        memcpy(&f, &v, 4);
        return f;
    };
    std::vector<Node2> roots(S);
    std::vector<Task> large0, small0;
    for (int i = 0; i < S; i++) {
        const uint32_t* a = &hacc[(size_t)i * 12];
        Node2& r = roots[i];
        Task t;
        t.node = i;
        t.start = seg[i];
        t.count = seg[i + 1] - seg[i];
        t.depth = 0;
        for (int k = 0; k < 3; k++) {
            r.lo[k] = ordf(a[k]);
            r.hi[k] = ordf(a[3 + k]);
            t.clo[k] = ordf(a[6 + k]);
            t.chi[k] = ordf(a[9 + k]);
        }
        r.a = 0;
        r.b = 0;
        if (t.count <= cfg.max_leaf) {
            r.a = t.start;
            r.b = -t.count;
        } else if (t.count <= cfg.small_task) {
            small0.push_back(t);
        } else {
            large0.push_back(t);
        }
    }
    if (!RT_CUDA(cudaMemcpyAsync(out.nodes.p, roots.data(), roots.size() * sizeof(Node2), cudaMemcpyHostToDevice, s)))
        return false;
    if (!large0.empty() &&
        !RT_CUDA(cudaMemcpyAsync(tasks_a.p, large0.data(), large0.size() * sizeof(Task), cudaMemcpyHostToDevice, s)))
        return false;
    if (!small0.empty() &&
        !RT_CUDA(cudaMemcpyAsync(small.p, small0.data(), small0.size() * sizeof(Task), cudaMemcpyHostToDevice, s)))
        return false;
    int num_small = (int)small0.size();
    int* d_small_base = flags.p + 8 * maxT;  // running count of small tasks
    int* d_tot = d_small_base + 1;           // scratch totals [large, small, chunks]
    int* d_C = d_tot + 2;
    // ctl: [0] this level's task count, [1] next node id, [2 + l] task count
    // of level l + 1 as logged for the host
    TmpBuf<int> ctl;
    if (!ctl.alloc(2 + kMaxLevels, s)) return false;
    int* d_T = ctl.p;
    int* d_node = ctl.p + 1;
    const int init[2] = {(int)large0.size(), S};
    if (!RT_CUDA(cudaMemcpyAsync(d_small_base, &num_small, sizeof(int), cudaMemcpyHostToDevice, s)) ||
        !RT_CUDA(cudaMemcpyAsync(ctl.p, init, sizeof(init), cudaMemcpyHostToDevice, s)) ||
        !RT_CUDA(cudaStreamSynchronize(s)))
        return false;
    Task* cur = tasks_a.p;
    Task* nxt = tasks_b.p;
    int* is_large = flags.p;
    int* is_small = flags.p + 2 * maxT;
    int* large_off = flags.p + 4 * maxT;
    int* small_off = flags.p + 6 * maxT;
    // Levels are queued ahead of the host: every launch is sized for an
    // upper bound (a level has at most twice the tasks of the one before,
    // and at most maxT), and the host learns each level's count one level
    // later, while the GPU already works on the next.  A level queued after
    // the last real one has no tasks and does nothing.
    LevelLog* lg = level_log();
    if (!lg) return false;
    int Tb = (int)large0.size();
    for (int lvl = 0; Tb > 0; lvl++) {
        if (lvl >= kMaxLevels) {
            set_error("build: more than %d levels", kMaxLevels);
            return false;
        }
        const int Cb = n / CHUNK + Tb + 1;  // sum over tasks of ceil(count / CHUNK) <= n / CHUNK + T
        const int Kb = 2 * Tb;
        k_chunk_counts<<<(Tb + 255) / 256, 256, 0, s>>>(cur, d_T, Tb, ccount.p);
        if (!scan_exclusive(ccount.p, coff.p, Tb, d_C, s)) return false;
        k_fill_chunks<<<Tb, 128, 0, s>>>(cur, d_T, coff.p, chunks.p);
        k_clear_bins<<<std::min(Tb * 8, 4096), 256, 0, s>>>(gbins.p, d_T);
        k_bin_large<<<Cb, CHUNK_T, 0, s>>>(chunks.p, cur, perm, d_lo, d_hi, gbins.p, d_C);
        k_split_large<<<(Tb + 3) / 4, 128, 0, s>>>(cur, d_T, gbins.p, splits.p, kids.p, kcb.p, out.nodes.p, d_node,
                                                    cfg.max_leaf, cfg.max_sah_depth);
        k_count_left<<<Cb, CHUNK_T, 0, s>>>(chunks.p, cur, splits.p, perm, d_lo, d_hi, cleft.p, kcb.p, d_C, side.p);
        if (!scan_exclusive(cleft.p, cleftoff.p, Cb, nullptr, s)) return false;
        k_scatter<<<Cb, CHUNK_T, 0, s>>>(chunks.p, cur, splits.p, perm, side.p, cleftoff.p, tmp.p, d_C);
        k_copy_back<<<Cb, 256, 0, s>>>(chunks.p, tmp.p, perm, d_C);
        k_classify_flags<<<(Kb + 255) / 256, 256, 0, s>>>(kids.p, d_T, Kb, cfg.max_leaf, cfg.small_task, is_large,
                                                          is_small);
        if (!scan_exclusive(is_large, large_off, Kb, d_tot, s)) return false;
        if (!scan_exclusive(is_small, small_off, Kb, d_tot + 1, s)) return false;
        k_compact_kids<<<(Kb + 255) / 256, 256, 0, s>>>(kids.p, d_T, is_large, large_off, is_small, small_off, nxt,
                                                        maxT, small.p, maxSmall, d_small_base, kcb.p, status.p);
        k_level_end<<<1, 1, 0, s>>>(d_T, d_node, d_small_base, d_tot, maxT, maxSmall, ctl.p + 2 + lvl, status.p);
        if (!RT_CUDA(cudaMemcpyAsync(lg->count + lvl, ctl.p + 2 + lvl, sizeof(int), cudaMemcpyDeviceToHost, s)) ||
            !RT_CUDA(cudaEventRecord(lg->ev[lvl], s)))
            return false;
        std::swap(cur, nxt);
        Tb = std::min(2 * Tb, maxT);
        if (lvl >= 1) {
            if (!RT_CUDA(cudaEventSynchronize(lg->ev[lvl - 1]))) return false;
            if (lg->count[lvl - 1] == 0) Tb = 0;  // this level had no tasks: done
        }
    }
    int hc[2] = {0, 0};
    if (!RT_CUDA(cudaMemcpyAsync(&hc[0], d_node, sizeof(int), cudaMemcpyDeviceToHost, s)) ||
        !RT_CUDA(cudaMemcpyAsync(&hc[1], d_small_base, sizeof(int), cudaMemcpyDeviceToHost, s)) ||
        !RT_CUDA(cudaStreamSynchronize(s)))
        return false;
    int node_count = hc[0];
    num_small = hc[1];
    if (num_small > 0) {
        TmpBuf<int> need, off;
        if (!need.alloc(num_small, s) || !off.alloc(num_small, s)) return false;
        k_reserve<<<(num_small + 255) / 256, 256, 0, s>>>(small.p, num_small, need.p);
        if (!scan_exclusive(need.p, off.p, num_small, d_tot, s)) return false;
        int reserved = 0;
        cudaMemcpyAsync(&reserved, d_tot, sizeof(int), cudaMemcpyDeviceToHost, s);
        // subtrees of at most warp_task primitives: one warp each (tasks hold
        // more than max_leaf primitives, so at most n / (max_leaf + 1) of them)
        const int warp_task = std::min(cfg.warp_task, WARP_TASK);
        const int wq_cap = warp_task > 0 ? n / (cfg.max_leaf + 1) + 2 : 0;
        TmpBuf<WTask> wq;
        if (wq_cap > 0 && !wq.alloc(wq_cap, s)) return false;
        int* d_wq_count = d_tot + 1;
        cudaMemsetAsync(d_wq_count, 0, sizeof(int), s);
        const size_t smem = (size_t)cfg.small_task * (6 * 4 + 4 + 2 + 2) + 16 + 3 * kBins * 7 * 4;
        cudaFuncSetAttribute(k_build_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_build_small<<<num_small, SMALL_T, smem, s>>>(small.p, off.p, node_count, perm, d_lo, d_hi, out.nodes.p,
                                                       cfg.max_leaf, cfg.max_sah_depth, cfg.small_task, warp_task,
                                                       wq.p, wq_cap, d_wq_count, status.p);
        if (warp_task > 0) {
            static const int grid = [] {  // persistent: as many CTAs as fit
                int per_sm = 0;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_build_warp, WB_T, 0) != cudaSuccess) {
                    cudaGetLastError();
                    per_sm = 1;
                }
                return num_sms() * std::max(per_sm, 1);
            }();
            k_build_warp<<<grid, WB_T, 0, s>>>(wq.p, d_wq_count, wq_cap, perm, d_lo, d_hi, out.nodes.p, cfg.max_leaf,
                                               cfg.max_sah_depth);
        }
        if (!RT_CUDA(cudaStreamSynchronize(s))) return false;
        node_count += reserved;
    }
    int st = 0;
    cudaMemcpyAsync(&st, status.p, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!RT_CUDA(cudaStreamSynchronize(s))) return false;
    if (st) {
        set_error("build: %s", (st & 8) ? "task list overflow" : (st & 2) ? "subtree queue overflow"
                                                                        : "subtree stack overflow");
        return false;
    }
    out.num_nodes = node_count;
    return true;
}


// ------------------------------------------------- graph-driven build --
// The whole build -- per-scene roots, the level loop of large tasks, the
// small and warp tiers, and the 8-wide collapse -- enqueued as ONE CUDA
// graph whose two level loops are conditional WHILE nodes: no count ever
// travels to the host, grids are sized for upper bounds (threads past the
// device's counts exit, as in the host-driven loop), and the result is the
// same tree, node for node.
struct BuildCtl {
    int T;         // this level's large-task count
    int node;      // next free binary node id
    int small;     // small tasks so far
    int tot[2];    // scan totals: large and small kids of the level
    int C;         // chunks of the level
    int levels;    // levels run
    int log_T;     // (k_level_end's per-level log slot, unused here)
    int reserved;  // node ids reserved by the small tasks
    int wq_count;  // warp-task queue length
    int work;      // small-task work counter
    int status;    // as the host-driven build; 16: more than kMaxLevels levels
};

__global__ void k_acc_init(uint32_t* __restrict__ acc, int S) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 12 * S; i += gridDim.x * blockDim.x) {
        const int k = i % 12;
        acc[i] = ((k >= 3 && k < 6) || k >= 9) ? 0u : 0xFFFFFFFFu;
    }
}

// One CTA: every segment's root node and task, in segment order (leaf
// roots finish here; the others go to the large or small task list), the
// counters, and the loop condition.
constexpr int ROOTS_T = 256;
__global__ void __launch_bounds__(ROOTS_T) k_roots(const uint32_t* __restrict__ acc, const int* __restrict__ seg, int S,
                                                   int max_leaf, int small_task, Node2* __restrict__ nodes,
                                                   Task* __restrict__ large, Task* __restrict__ small,
                                                   BuildCtl* __restrict__ ctl, cudaGraphConditionalHandle cond) {
    __shared__ int ws[ROOTS_T / 32];
    int nl = 0, ns = 0;
    for (int base = 0; base < S; base += ROOTS_T) {
        const int i = base + threadIdx.x;
        Task t = {};
        Node2 r = {};
        int is_l = 0, is_s = 0;
        if (i < S) {
            const uint32_t* a = acc + (size_t)i * 12;
            t.node = i;
            t.start = seg[i];
            t.count = seg[i + 1] - seg[i];
            t.depth = 0;
            for (int k = 0; k < 3; k++) {
                r.lo[k] = ord2f(a[k]);
                r.hi[k] = ord2f(a[3 + k]);
                t.clo[k] = ord2f(a[6 + k]);
                t.chi[k] = ord2f(a[9 + k]);
            }
            if (t.count <= max_leaf) {
                r.a = t.start;
                r.b = -t.count;
            } else if (t.count <= small_task) {
                is_s = 1;
            } else {
                is_l = 1;
            }
            nodes[i] = r;
        }
        int tl, ts;
        const int ol = block_exclusive_scan<ROOTS_T>(is_l, ws, tl);
        const int os = block_exclusive_scan<ROOTS_T>(is_s, ws, ts);
        if (is_l) large[nl + ol] = t;
        if (is_s) small[ns + os] = t;
        nl += tl;
        ns += ts;
    }
    if (threadIdx.x == 0) {
        BuildCtl c = {};
        c.T = nl;
        c.node = S;
        c.small = ns;
        *ctl = c;
        cudaGraphSetConditional(cond, nl > 0 ? 1u : 0u);
    }
}

// After k_level_end: the next level's tasks become the current ones (the
// loop's kernels keep fixed buffer arguments), and the loop goes on while
// tasks remain, nothing overflowed and the level bound holds.
__global__ void k_level_next(const Task* __restrict__ nxt, Task* __restrict__ cur, BuildCtl* __restrict__ ctl,
                             cudaGraphConditionalHandle cond) {
    const int T = ctl->T;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) cur[i] = nxt[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int lv = ++ctl->levels;
        if (T > 0 && lv >= kMaxLevels) ctl->status |= 16;
        cudaGraphSetConditional(cond, (T > 0 && lv < kMaxLevels && !(ctl->status & 8)) ? 1u : 0u);
    }
}

// Node ids each small task reserves (2 count - 2), zero past the count.
__global__ void k_reserve_n(const Task* __restrict__ small, const int* __restrict__ d_S, int cap,
                            int* __restrict__ need) {
    const int S = *d_S;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x)
        need[i] = i < S ? 2 * small[i].count - 2 : 0;
}

__global__ void k_build_result(const BuildCtl* __restrict__ ctl, int* __restrict__ out) {
    out[0] = ctl->node + ctl->reserved;
    out[1] = ctl->status;
    out[2] = ctl->levels;
    out[3] = ctl->small;
}

bool graph_build_supported() {
    // conditional WHILE nodes and capture into a node's body graph: CUDA 12.4
    static const bool ok = [] {
        int v = 0;
        if (cudaDriverGetVersion(&v) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return v >= 12040;
    }();
    return ok;
}

bool build_bvh8_graph(const float4* d_lo, const float4* d_hi, const float* d_tris9, int n, const BuildConfig& cfg,
                      const std::vector<int>& seg, Bvh8Device& out, cudaStream_t s, GraphBuildInfo* info,
                      Bvh2Device* keep) {
    GraphBuildJob job;
    return launch_bvh8_graph(d_lo, d_hi, d_tris9, n, cfg, seg, out, s, job, keep) && finish_bvh8_graph(job, info);
}

// A build's segment table from absolute offsets already on the device.
__global__ void k_seg_rebase(const int* __restrict__ src, int count, int base, int* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) dst[i] = src[i] - base;
}

bool launch_bvh8_graph(const float4* d_lo, const float4* d_hi, const float* d_tris9, int n, const BuildConfig& cfg,
                       const std::vector<int>& seg, Bvh8Device& out, cudaStream_t s, GraphBuildJob& job,
                       Bvh2Device* keep, const int* d_seg, int seg_base) {
    if (job.launched) {
        set_error("graph build: job already launched");
        return false;
    }
    if (n <= 0 || !d_tris9) {
        set_error("graph build: empty input");
        return false;
    }
    if (cfg.max_leaf < 1 || cfg.max_leaf > 4 || cfg.small_task < WARP_TASK || cfg.small_task > 32 * SMALL_T) {
        set_error("graph build: bad configuration");
        return false;
    }
    const int S = (int)seg.size() - 1;
    if (S < 1 || seg.front() != 0 || seg.back() != n) {
        set_error("graph build: bad segment table");
        return false;
    }
    if (S > kMaxSegments) {
        set_error("graph build: %d scenes, at most %d per build", S, kMaxSegments);
        return false;
    }
    int maxcnt = 0;
    for (int i = 0; i < S; i++) {
        if (seg[i + 1] <= seg[i]) {
            set_error("graph build: segment %d is empty", i);
            return false;
        }
        maxcnt = std::max(maxcnt, seg[i + 1] - seg[i]);
    }
    // upper bounds the graph's grids and buffers are sized for
    const int maxT = n / (cfg.small_task + 1) + 2;     // large tasks per level
    const int Cb = n / CHUNK + maxT + 1;               // chunks per level
    const int maxChunks = Cb + 1;
    const int Kb = 2 * maxT;                           // kids per level
    const int maxSmall = n / (cfg.max_leaf + 1) + 2;   // small tasks in all
    const int slots = 2 * n + 2;                       // binary node ids
    const int warp_task = std::min(cfg.warp_task, WARP_TASK);
    const int wq_cap = warp_task > 0 ? n / (cfg.max_leaf + 1) + 2 : 0;
    const int scan_cap = std::max(std::max(maxT, Cb), std::max(Kb, maxSmall));
    const size_t cbytes = collapse_graph_scratch_bytes(n, S, slots, true);
    TmpBuf<Node2> tnodes;
    TmpBuf<int> tperm, tmp, dseg, ccount, coff, cleft, cleftoff, flags, need, off, scan;
    TmpBuf<int>& result = job.result;
    TmpBuf<uint32_t> acc, gbins, kcb;
    TmpBuf<Task> tasks_a, tasks_b, kids, small;
    TmpBuf<Split> splits;
    TmpBuf<uint8_t> side;
    TmpBuf<Chunk> chunks;
    TmpBuf<WTask> wq;
    TmpBuf<BuildCtl> ctl;
    TmpBuf<char> cscratch;
    // the binary tree: scratch, or the caller's (kept for exports and refits)
    if (keep ? (!keep->nodes.alloc(slots) || !keep->perm.alloc(n)) : (!tnodes.alloc(slots, s) || !tperm.alloc(n, s)))
        return false;
    Node2* d_nodes = keep ? keep->nodes.p : tnodes.p;
    int* d_perm = keep ? keep->perm.p : tperm.p;
    if (!tmp.alloc(n, s) || !dseg.alloc(S + 1, s) ||
        !acc.alloc((size_t)12 * S, s) || !tasks_a.alloc(maxT, s) || !tasks_b.alloc(maxT, s) || !kids.alloc(Kb, s) ||
        !small.alloc(maxSmall, s) || !splits.alloc(maxT, s) || !gbins.alloc((size_t)maxT * TASK_BIN_WORDS, s) ||
        !flags.alloc((size_t)4 * Kb, s) || !kcb.alloc((size_t)12 * maxT, s) || !side.alloc(n, s) ||
        !chunks.alloc(maxChunks, s) || !ccount.alloc(maxT, s) || !coff.alloc(maxT, s) || !cleft.alloc(maxChunks, s) ||
        !cleftoff.alloc(maxChunks, s) || !need.alloc(maxSmall, s) || !off.alloc(maxSmall, s) ||
        (wq_cap > 0 && !wq.alloc(wq_cap, s)) || !ctl.alloc(1, s) || !scan.alloc(scan_scratch_ints(scan_cap), s) ||
        !result.alloc(8, s) || !cscratch.alloc(cbytes, s))
        return false;
    // the output: a caller's buffers when large enough (pooled group
    // outputs of a batch build), else allocated here
    if (!out.nodes.ensure((size_t)n + S) || !out.tris.ensure(n)) return false;
    if (d_seg) {
        k_seg_rebase<<<(S + 1 + 255) / 256, 256, 0, s>>>(d_seg, S + 1, seg_base, dseg.p);
        if (!RT_CUDA(cudaGetLastError())) return false;
    } else if (!RT_CUDA(cudaMemcpyAsync(dseg.p, seg.data(), sizeof(int) * (S + 1), cudaMemcpyHostToDevice, s))) {
        return false;
    }
    const size_t smem = (size_t)cfg.small_task * (6 * 4 + 4 + 2 + 2) + 16 + 3 * kBins * 7 * 4;
    if (!RT_CUDA(cudaFuncSetAttribute(k_build_small_loop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
        return false;
    int small_per_sm = 0, warp_per_sm = 0;
    if (!RT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&small_per_sm, k_build_small_loop, SMALL_T, smem)) ||
        !RT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&warp_per_sm, k_build_warp, WB_T, 0)))
        return false;
    const int small_grid = num_sms() * std::max(1, small_per_sm);
    const int warp_grid = num_sms() * std::max(1, warp_per_sm);

    // capture on two private streams; nothing runs until the launch on s
    cudaStream_t cs = nullptr, bs = nullptr;
    if (!RT_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) ||
        !RT_CUDA(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking))) {
        if (cs) cudaStreamDestroy(cs);
        return false;
    }
    cudaGraph_t graph = nullptr;
    bool ok = RT_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed));
    bool capturing = ok;
    BuildCtl* c = ctl.p;
    Task* cur = tasks_a.p;
    Task* nxt = tasks_b.p;
    int* is_large = flags.p;
    int* is_small = flags.p + Kb;
    int* large_off = flags.p + 2 * Kb;
    int* small_off = flags.p + 3 * Kb;
    if (ok) {
        cudaMemsetAsync(d_nodes, 0, sizeof(Node2) * (size_t)slots, cs);
        k_iota<<<(n + 255) / 256, 256, 0, cs>>>(d_perm, n);
        k_acc_init<<<std::max(1, std::min((12 * S + 255) / 256, 1024)), 256, 0, cs>>>(acc.p, S);
        k_seg_bounds<<<dim3(std::min((maxcnt + 2047) / 2048, 64), S), 256, 0, cs>>>(d_lo, d_hi, dseg.p, acc.p);
        cudaGraphConditionalHandle lv_cond;
        cudaGraph_t body;
        ok = capture_conditional_handle(cs, &lv_cond);
        if (ok) {
            k_roots<<<1, ROOTS_T, 0, cs>>>(acc.p, dseg.p, S, cfg.max_leaf, cfg.small_task, d_nodes, cur, small.p, c,
                                           lv_cond);
            ok = capture_while(cs, lv_cond, &body) &&
                 RT_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        }
        if (ok) {
            // one level of large tasks (the host-driven loop's sequence)
            k_chunk_counts<<<(maxT + 255) / 256, 256, 0, bs>>>(cur, &c->T, maxT, ccount.p);
            bool lok = scan_exclusive_dev(ccount.p, coff.p, maxT, nullptr, &c->C, scan.p, bs);
            k_fill_chunks<<<maxT, 128, 0, bs>>>(cur, &c->T, coff.p, chunks.p);
            k_clear_bins<<<std::min(maxT * 8, 4096), 256, 0, bs>>>(gbins.p, &c->T);
            k_bin_large<<<Cb, CHUNK_T, 0, bs>>>(chunks.p, cur, d_perm, d_lo, d_hi, gbins.p, &c->C);
            k_split_large<<<(maxT + 3) / 4, 128, 0, bs>>>(cur, &c->T, gbins.p, splits.p, kids.p, kcb.p, d_nodes,
                                                          &c->node, cfg.max_leaf, cfg.max_sah_depth);
            k_count_left<<<Cb, CHUNK_T, 0, bs>>>(chunks.p, cur, splits.p, d_perm, d_lo, d_hi, cleft.p, kcb.p, &c->C,
                                                 side.p);
            lok = lok && scan_exclusive_dev(cleft.p, cleftoff.p, Cb, nullptr, nullptr, scan.p, bs);
            k_scatter<<<Cb, CHUNK_T, 0, bs>>>(chunks.p, cur, splits.p, d_perm, side.p, cleftoff.p, tmp.p, &c->C);
            k_copy_back<<<Cb, 256, 0, bs>>>(chunks.p, tmp.p, d_perm, &c->C);
            k_classify_flags<<<(Kb + 255) / 256, 256, 0, bs>>>(kids.p, &c->T, Kb, cfg.max_leaf, cfg.small_task,
                                                               is_large, is_small);
            lok = lok && scan_exclusive_dev(is_large, large_off, Kb, nullptr, &c->tot[0], scan.p, bs) &&
                  scan_exclusive_dev(is_small, small_off, Kb, nullptr, &c->tot[1], scan.p, bs);
            k_compact_kids<<<(Kb + 255) / 256, 256, 0, bs>>>(kids.p, &c->T, is_large, large_off, is_small, small_off,
                                                             nxt, maxT, small.p, maxSmall, &c->small, kcb.p,
                                                             &c->status);
            k_level_end<<<1, 1, 0, bs>>>(&c->T, &c->node, &c->small, c->tot, maxT, maxSmall, &c->log_T, &c->status);
            k_level_next<<<std::min((maxT + 255) / 256, 1024), 256, 0, bs>>>(nxt, cur, c, lv_cond);
            lok = lok && RT_CUDA(cudaGetLastError());
            cudaGraph_t done = nullptr;
            ok = RT_CUDA(cudaStreamEndCapture(bs, &done)) && lok;
        }
        if (ok) {
            // small tasks (one CTA each, persistent) and warp subtrees
            k_reserve_n<<<std::min((maxSmall + 255) / 256, num_sms() * 16), 256, 0, cs>>>(small.p, &c->small,
                                                                                          maxSmall, need.p);
            ok = scan_exclusive_dev(need.p, off.p, maxSmall, &c->small, &c->reserved, scan.p, cs);
            k_build_small_loop<<<small_grid, SMALL_T, smem, cs>>>(small.p, &c->small, &c->work, off.p, &c->node,
                                                                  d_perm, d_lo, d_hi, d_nodes, cfg.max_leaf,
                                                                  cfg.max_sah_depth, cfg.small_task, warp_task, wq.p,
                                                                  wq_cap, &c->wq_count, &c->status);
            if (warp_task > 0)
                k_build_warp<<<warp_grid, WB_T, 0, cs>>>(wq.p, &c->wq_count, wq_cap, d_perm, d_lo, d_hi, d_nodes,
                                                         cfg.max_leaf, cfg.max_sah_depth);
            k_build_result<<<1, 1, 0, cs>>>(c, result.p);
            ok = ok && RT_CUDA(cudaGetLastError());
        }
        ok = ok && enqueue_collapse_graph(d_nodes, d_perm, n, S, slots, d_tris9, out.nodes.p, out.tris.p, nullptr,
                                          cscratch.p, cbytes, result.p + 4, cs, bs);
        cudaGraph_t g = nullptr;
        const bool ended = RT_CUDA(cudaStreamEndCapture(cs, &g));
        capturing = false;
        graph = g;
        ok = ok && ended && graph;
    }
    if (capturing) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cs, &g);
        if (g) cudaGraphDestroy(g);
    }
    if (ok)
        ok = RT_CUDA(cudaEventCreate(&job.e0)) && RT_CUDA(cudaEventCreate(&job.e1)) &&
             RT_CUDA(cudaGraphInstantiate(&job.exec, graph, 0)) && RT_CUDA(cudaEventRecord(job.e0, s)) &&
             RT_CUDA(cudaGraphLaunch(job.exec, s)) && RT_CUDA(cudaEventRecord(job.e1, s));
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(bs);
    cudaStreamDestroy(cs);
    if (!ok) return false;
    job.s = s;
    job.n = n;
    job.S = S;
    job.out = &out;
    job.keep = keep;
    job.launched = true;
    return true;
}

bool finish_bvh8_graph(GraphBuildJob& job, GraphBuildInfo* info) {
    if (!job.launched) {
        set_error("graph build: nothing launched");
        return false;
    }
    job.launched = false;
    int h[8] = {};
    if (!RT_CUDA(cudaMemcpyAsync(h, job.result.p, sizeof(h), cudaMemcpyDeviceToHost, job.s)) ||
        !RT_CUDA(cudaStreamSynchronize(job.s)))
        return false;
    if (info) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, job.e0, job.e1);
        info->graph_ms = ms;
    }
    if (h[1]) {
        set_error("graph build: %s", (h[1] & 16) ? "more levels than the bound"
                                     : (h[1] & 8) ? "task list overflow"
                                     : (h[1] & 2) ? "subtree queue overflow"
                                                  : "subtree stack overflow");
        return false;
    }
    if (h[7]) {
        set_error("collapse: %s", (h[7] & 1) ? "capacity exceeded" : "more levels than the bound");
        return false;
    }
    Bvh8Device& out = *job.out;
    Bvh2Device* keep = job.keep;
    const int n = job.n, S = job.S;
    out.num_nodes = h[4];
    out.num_leaf_items = h[5];
    out.depth = h[6];
    if (keep) {
        keep->num_nodes = h[0];
        keep->num_prims = n;
        keep->num_roots = S;
    }
    if (info) {
        info->bvh2_nodes = h[0];
        info->levels = h[2];
        info->small_tasks = h[3];
    }
    return true;
}

}  // namespace rtb
