// rt_geometry.cu -- BLAS construction from the application's own vertex and
// index buffers, refit after vertex animation, and a versioned BVH blob.
//
//   cudaBVH_buildGeometries   The reference layer reads every BLAS's vertex
//                             and index buffers back to the host and rebuilds
//                             a triangle soup there (layer/VkLayer_CudaRT.cpp:
//                             2961-2981, 3087-3125).  Here one kernel gathers
//                             the triangles on the device (float3 or half3
//                             vertices at any stride, uint16 / uint32 / no
//                             indices, an optional 3x4 transform) and the GPU
//                             builder runs on them; nothing crosses PCIe.
//   cudaBVH_refit             New vertex positions, same triangles in the same
//                             order: the binary BVH's boxes are recomputed
//                             bottom-up (one thread per leaf walks to the root;
//                             the second child to arrive at a node computes
//                             its box) and the 8-wide layout is re-emitted.
//                             The topology is kept, so quality degrades with
//                             large motion; rebuild when the SAH cost grows.
//   cudaBVH_serialize /       A host blob: header (magic, version, counts,
//   cudaBVH_deserialize       bounds, statistics, 64-bit checksum of the
//                             payload) then the input triangles, the binary
//                             BVH with its permutation, the 8-wide nodes and
//                             the triangle records, each 16-byte aligned.
//                             Loading is one upload per section, no build.
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include <cuda/atomic>

#include "rt_internal.h"

using namespace rtb;

namespace {

struct Xform {
    float m[12];
};

__device__ __forceinline__ float vcomp(const char* base, int fmt, int c) {
    if (fmt == RT_VERTEX_HALF3) {
        unsigned short u = reinterpret_cast<const unsigned short*>(base)[c];
        return __half2float(__ushort_as_half(u));
    }
    return reinterpret_cast<const float*>(base)[c];
}

// Gathers num triangles of one geometry into out (9 floats each).  Indices
// above max_vertex are not followed: the triangle is written degenerate and
// *bad is set, which makes the build fail.
__global__ void k_gather_geometry(const char* __restrict__ verts, unsigned long long stride, int fmt,
                                  const void* __restrict__ idx, int itype, int num, int max_vertex, Xform x,
                                  int has_x, float* __restrict__ out, int* __restrict__ bad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= num) return;
    unsigned int vi[3];
    for (int k = 0; k < 3; k++) {
        if (itype == RT_INDEX_UINT16) vi[k] = reinterpret_cast<const unsigned short*>(idx)[3 * (size_t)p + k];
        else if (itype == RT_INDEX_UINT32) vi[k] = reinterpret_cast<const unsigned int*>(idx)[3 * (size_t)p + k];
        else vi[k] = 3u * (unsigned int)p + (unsigned int)k;
    }
    float* o = out + (size_t)p * 9;
    if (vi[0] > (unsigned)max_vertex || vi[1] > (unsigned)max_vertex || vi[2] > (unsigned)max_vertex) {
        for (int k = 0; k < 9; k++) o[k] = 0.f;
        atomicOr(bad, 1);
        return;
    }
    for (int k = 0; k < 3; k++) {
        const char* v = verts + (size_t)vi[k] * stride;
        const float a = vcomp(v, fmt, 0), b = vcomp(v, fmt, 1), c = vcomp(v, fmt, 2);
        if (has_x) {
            // row r: ((m[4r] a + m[4r+1] b) + m[4r+2] c) + m[4r+3], each step rounded
            for (int r = 0; r < 3; r++)
                o[3 * k + r] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x.m[4 * r], a), __fmul_rn(x.m[4 * r + 1], b)),
                                                   __fmul_rn(x.m[4 * r + 2], c)),
                                         x.m[4 * r + 3]);
        } else {
            o[3 * k] = a;
            o[3 * k + 1] = b;
            o[3 * k + 2] = c;
        }
    }
}

// Checks the descriptions and gathers every geometry into d_out (device,
// 9 floats per triangle, geometries back to back); false with the error set.
bool gather_geometries(const RtGeometry* g, int ng, float* d_out, int* d_bad, cudaStream_t s, const char* who) {
    size_t off = 0;
    for (int i = 0; i < ng; i++) {
        const RtGeometry& q = g[i];
        const size_t esz = q.vertex_format == RT_VERTEX_HALF3 ? 2 : 4;
        const bool fmt_ok = q.vertex_format == RT_VERTEX_FLOAT3 || q.vertex_format == RT_VERTEX_HALF3;
        const bool idx_ok = q.index_type == RT_INDEX_NONE || q.index_type == RT_INDEX_UINT16 ||
                            q.index_type == RT_INDEX_UINT32;
        if (!fmt_ok || !idx_ok || !q.d_vertices || q.num_triangles < 0 || q.max_vertex < 0 ||
            q.vertex_stride < 3 * esz || (q.vertex_stride % esz) != 0 || misaligned(q.d_vertices, esz) ||
            (q.index_type != RT_INDEX_NONE && !q.d_indices) ||
            misaligned(q.d_indices, q.index_type == RT_INDEX_UINT16 ? 2 : 4)) {
            set_error("%s: geometry %d: invalid description (format, stride, alignment or buffers)", who, i);
            return false;
        }
        if (q.index_type == RT_INDEX_NONE && 3ll * q.num_triangles - 1 > (long long)q.max_vertex) {
            set_error("%s: geometry %d: %d non-indexed triangles need vertices up to %lld > max_vertex %d", who, i,
                      q.num_triangles, 3ll * q.num_triangles - 1, q.max_vertex);
            return false;
        }
        if (q.num_triangles == 0) continue;
        Xform x{};
        if (q.transform) memcpy(x.m, q.transform, sizeof(x.m));
        k_gather_geometry<<<(q.num_triangles + 255) / 256, 256, 0, s>>>(
            reinterpret_cast<const char*>(q.d_vertices), q.vertex_stride, q.vertex_format, q.d_indices, q.index_type,
            q.num_triangles, q.max_vertex, x, q.transform ? 1 : 0, d_out + off * 9, d_bad);
        off += (size_t)q.num_triangles;
    }
    int bad = 0;
    if (!RT_CUDA(cudaGetLastError()) ||
        !RT_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s)) ||
        !RT_CUDA(cudaStreamSynchronize(s)))
        return false;
    if (bad) {
        set_error("%s: an index exceeds max_vertex", who);
        return false;
    }
    return true;
}

long long total_triangles(const RtGeometry* g, int ng) {
    long long n = 0;
    for (int i = 0; i < ng; i++) n += g[i].num_triangles > 0 ? g[i].num_triangles : 0;
    return n;
}

// ---- refit ----
__global__ void k_parents(const Node2* __restrict__ nodes, int slots, int* __restrict__ parent,
                          int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= slots) return;
    const Node2 nd = nodes[i];
    if (nd.b > 0) {  // inner node (unused reserved slots have b == 0)
        if (nd.a <= 0 || nd.a >= slots || nd.b >= slots) {
            atomicOr(status, 2);  // malformed tree: children out of range
            return;
        }
        parent[nd.a] = i;
        parent[nd.b] = i;
    }
}

// One thread per leaf: leaf box from the new triangle boxes, then up the
// tree; at every node the first arriving child stops and the second computes
// the node's box from both children (fence before the arrival counter, L2
// loads after it).  The walk is bounded by kMaxDepth steps.
constexpr int kMaxDepth = 256;
__global__ void k_refit(Node2* __restrict__ nodes, int slots, const int* __restrict__ parent,
                        const int* __restrict__ perm, int nprims, const float4* __restrict__ lo,
                        const float4* __restrict__ hi, int* __restrict__ arrive, int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= slots) return;
    const Node2 nd = nodes[i];
    if (nd.b >= 0) return;  // leaves only
    if (nd.a < 0 || (long long)nd.a - nd.b > nprims) {
        atomicOr(status, 2);  // malformed leaf range
        return;
    }
    float l0 = INFINITY, l1 = INFINITY, l2 = INFINITY, h0 = -INFINITY, h1 = -INFINITY, h2 = -INFINITY;
    for (int j = nd.a; j < nd.a - nd.b; j++) {
        const int p = perm[j];
        if (p < 0 || p >= nprims) {
            atomicOr(status, 2);
            return;
        }
        const float4 a = lo[p], b = hi[p];
        l0 = fminf(l0, a.x); l1 = fminf(l1, a.y); l2 = fminf(l2, a.z);
        h0 = fmaxf(h0, b.x); h1 = fmaxf(h1, b.y); h2 = fmaxf(h2, b.z);
    }
    nodes[i].lo[0] = l0; nodes[i].lo[1] = l1; nodes[i].lo[2] = l2;
    nodes[i].hi[0] = h0; nodes[i].hi[1] = h1; nodes[i].hi[2] = h2;
    int cur = i;
    for (int step = 0;; step++) {
        const int par = parent[cur];
        if (par < 0) return;
        if (step >= kMaxDepth) {
            atomicOr(status, 1);
            return;
        }
        // release our box, acquire the sibling's: the second arrival sees both
        cuda::atomic_ref<int, cuda::thread_scope_device> arr(arrive[par]);
        if (arr.fetch_add(1, cuda::memory_order_acq_rel) == 0) return;
        const int a = __ldcg(&nodes[par].a), b = __ldcg(&nodes[par].b);
        float bl[3], bh[3];
        for (int k = 0; k < 3; k++) {
            bl[k] = fminf(__ldcg(&nodes[a].lo[k]), __ldcg(&nodes[b].lo[k]));
            bh[k] = fmaxf(__ldcg(&nodes[a].hi[k]), __ldcg(&nodes[b].hi[k]));
        }
        for (int k = 0; k < 3; k++) {
            nodes[par].lo[k] = bl[k];
            nodes[par].hi[k] = bh[k];
        }
        cur = par;
    }
}

bool refit_handle(CudaBVHHandle* h, cudaStream_t s) {
    Bvh2Device& b2 = h->bvh2;
    const int n = h->num_tris, slots = b2.num_nodes;
    if (b2.num_roots != 1) {
        set_error("cudaBVH_refit: handle has %d roots", b2.num_roots);
        return false;
    }
    TmpBuf<float4> lo, hi;
    TmpBuf<int> parent, arrive, status;
    if (!lo.alloc(n, s) || !hi.alloc(n, s) || !parent.alloc(slots, s) || !arrive.alloc(slots, s) ||
        !status.alloc(1, s))
        return false;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    launch_tri_bounds(h->tris9.p, n, lo.p, hi.p, s);
    bool ok = RT_CUDA(cudaMemsetAsync(parent.p, 0xFF, sizeof(int) * (size_t)slots, s)) &&
              RT_CUDA(cudaMemsetAsync(arrive.p, 0, sizeof(int) * (size_t)slots, s)) &&
              RT_CUDA(cudaMemsetAsync(status.p, 0, sizeof(int), s));
    if (ok) {
        k_parents<<<(slots + 255) / 256, 256, 0, s>>>(b2.nodes.p, slots, parent.p, status.p);
        k_refit<<<(slots + 255) / 256, 256, 0, s>>>(b2.nodes.p, slots, parent.p, b2.perm.p, b2.num_prims, lo.p, hi.p,
                                                    arrive.p, status.p);
        ok = RT_CUDA(cudaGetLastError());
    }
    int st = 0;
    ok = ok && RT_CUDA(cudaMemcpyAsync(&st, status.p, sizeof(int), cudaMemcpyDeviceToHost, s)) &&
         RT_CUDA(cudaStreamSynchronize(s));
    if (ok && st) {
        set_error(st & 2 ? "cudaBVH_refit: malformed binary BVH" : "cudaBVH_refit: tree deeper than %d levels",
                  kMaxDepth);
        ok = false;
    }
    // re-emit the 8-wide layout; keep the buffers (and so the device pointers
    // a TLAS or a server may hold) when the new layout fits them
    Bvh8Device t;
    ok = ok && collapse_bvh8(b2, h->tris9.p, t, s);
    if (ok) {
        if (t.num_nodes <= (int)h->bvh8.nodes.n && t.num_leaf_items <= (int)h->bvh8.tris.n) {
            ok = RT_CUDA(cudaMemcpyAsync(h->bvh8.nodes.p, t.nodes.p, sizeof(Bvh8Node) * (size_t)t.num_nodes,
                                         cudaMemcpyDeviceToDevice, s)) &&
                 RT_CUDA(cudaMemcpyAsync(h->bvh8.tris.p, t.tris.p, sizeof(TriRec) * (size_t)t.num_leaf_items,
                                         cudaMemcpyDeviceToDevice, s));
        } else {
            std::swap(h->bvh8.nodes.p, t.nodes.p);
            std::swap(h->bvh8.nodes.n, t.nodes.n);
            std::swap(h->bvh8.tris.p, t.tris.p);
            std::swap(h->bvh8.tris.n, t.tris.n);
        }
        h->bvh8.num_nodes = t.num_nodes;
        h->bvh8.num_leaf_items = t.num_leaf_items;
        h->bvh8.depth = t.depth;
    }
    cudaEventRecord(e1, s);
    ok = ok && RT_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    if (ok) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!ok) return false;
    Node2 root;
    if (!RT_CUDA(cudaMemcpy(&root, b2.nodes.p, sizeof(Node2), cudaMemcpyDeviceToHost))) return false;
    for (int a = 0; a < 3; a++) {
        h->bmin[a] = root.lo[a];
        h->bmax[a] = root.hi[a];
        h->center[a] = (root.lo[a] + root.hi[a]) * 0.5f;
    }
    const float ex = h->bmax[0] - h->bmin[0], ey = h->bmax[1] - h->bmin[1], ez = h->bmax[2] - h->bmin[2];
    h->extent = sqrtf(ex * ex + ey * ey + ez * ez);
    h->stats.num_nodes = h->bvh8.num_nodes;
    h->stats.depth = h->bvh8.depth;
    h->stats.build_ms = ms;
    h->stats.sah_cost = bvh2_sah_cost(b2, s);
    h->stats.node_bytes = (uint64_t)h->bvh8.num_nodes * sizeof(Bvh8Node);
    h->exports_ready = false;
    if (getenv("RTB200_VALIDATE") && atoi(getenv("RTB200_VALIDATE")) &&
        !validate_bvh8(h->bvh8, h->bvh8.num_leaf_items, h->num_tris))
        return false;
    return true;
}

// ---- blob ----
constexpr char kMagic[8] = {'R', 'T', 'B', '2', '0', '0', 'B', 'V'};
constexpr uint32_t kVersion = 1;

struct BlobHeader {
    char magic[8];
    uint32_t version, header_bytes;
    uint64_t payload_bytes, checksum;
    int32_t num_tris, bvh2_slots, num_prims, num_nodes8, num_items8, depth8, reserved[2];
    float bmin[3], bmax[3];
    RtBuildStats stats;
};

size_t pad16(size_t x) { return (x + 15) & ~size_t(15); }

struct Sections {
    size_t tris, bvh2, perm, nodes8, items8, total;
};

Sections sections(const BlobHeader& b) {
    Sections s;
    s.tris = pad16((size_t)b.num_tris * sizeof(CudaTri));
    s.bvh2 = pad16((size_t)b.bvh2_slots * sizeof(Node2));
    s.perm = pad16((size_t)b.num_prims * sizeof(int));
    s.nodes8 = pad16((size_t)b.num_nodes8 * sizeof(Bvh8Node));
    s.items8 = pad16((size_t)b.num_items8 * sizeof(TriRec));
    s.total = s.tris + s.bvh2 + s.perm + s.nodes8 + s.items8;
    return s;
}

// 64-bit FNV-1a over 8-byte words (the payload is a multiple of 16 bytes).
uint64_t checksum(const unsigned char* p, size_t n) {
    uint64_t h = 0xcbf29ce484222325ull;
    for (size_t i = 0; i + 8 <= n; i += 8) {
        uint64_t w;
        memcpy(&w, p + i, 8);
        h = (h ^ w) * 0x100000001b3ull;
    }
    return h;
}

// Host check of a blob's binary BVH before anything walks it: from the root
// every node is reached once, children are in range, leaf ranges cover the
// permutation exactly once, and the permutation is one.
bool check_bvh2(const unsigned char* nodes_raw, int slots, const unsigned char* perm_raw, int nprims) {
    std::vector<Node2> nd((size_t)slots);
    memcpy(nd.data(), nodes_raw, sizeof(Node2) * (size_t)slots);
    std::vector<int> perm((size_t)nprims);
    memcpy(perm.data(), perm_raw, sizeof(int) * (size_t)nprims);
    std::vector<unsigned char> seen((size_t)slots, 0), used((size_t)nprims, 0), pseen((size_t)nprims, 0);
    for (int p : perm) {
        if (p < 0 || p >= nprims || pseen[p]) return false;
        pseen[p] = 1;
    }
    std::vector<int> stack{0};
    long long covered = 0;
    while (!stack.empty()) {
        const int i = stack.back();
        stack.pop_back();
        if (i < 0 || i >= slots || seen[i]) return false;
        seen[i] = 1;
        const Node2& n = nd[i];
        if (n.b < 0) {
            if (n.a < 0 || (long long)n.a - n.b > nprims) return false;
            for (int j = n.a; j < n.a - n.b; j++) {
                if (used[j]) return false;
                used[j] = 1;
            }
            covered += -n.b;
        } else if (n.b > 0) {
            stack.push_back(n.a);
            stack.push_back(n.b);
        } else {
            return false;  // the root or a child cannot be an unused slot
        }
    }
    return covered == nprims;
}

}  // namespace

extern "C" {

CudaBVH_t cudaBVH_buildGeometries(const RtGeometry* geoms, int num_geoms, void* stream) {
    clear_error();
    if (!geoms || num_geoms <= 0) {
        set_error("cudaBVH_buildGeometries: invalid argument");
        return nullptr;
    }
    const long long n = total_triangles(geoms, num_geoms);
    if (n <= 0 || n > 0x7FFFFFFFll) {
        set_error("cudaBVH_buildGeometries: %lld triangles", n);
        return nullptr;
    }
    cudaStream_t s = (cudaStream_t)stream;
    CudaBVHHandle* h = create_handle((int)n);
    if (!h) return nullptr;
    TmpBuf<int> bad;
    const bool ok = h->tris9.alloc((size_t)n * 9) && bad.alloc(1, s) &&
                    RT_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s)) &&
                    gather_geometries(geoms, num_geoms, h->tris9.p, bad.p, s, "cudaBVH_buildGeometries") &&
                    build_handle(h, s);
    if (!ok) {
        delete h;
        return nullptr;
    }
    return h;
}

int cudaBVH_refit(CudaBVH_t h, const CudaTri* d_tris, void* stream) {
    clear_error();
    if (!h || !d_tris || misaligned(d_tris, 4)) {
        set_error("cudaBVH_refit: invalid argument");
        return RT_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    std::lock_guard<std::mutex> g(h->mu);
    if (!RT_CUDA(cudaMemcpyAsync(h->tris9.p, d_tris, sizeof(CudaTri) * (size_t)h->num_tris,
                                 cudaMemcpyDeviceToDevice, s)))
        return RT_ERR_CUDA;
    return refit_handle(h, s) ? RT_OK : RT_ERR_CUDA;
}

int cudaBVH_refitGeometries(CudaBVH_t h, const RtGeometry* geoms, int num_geoms, void* stream) {
    clear_error();
    if (!h || !geoms || num_geoms <= 0) {
        set_error("cudaBVH_refitGeometries: invalid argument");
        return RT_ERR_INVALID;
    }
    if (total_triangles(geoms, num_geoms) != h->num_tris) {
        set_error("cudaBVH_refitGeometries: %lld triangles, the handle has %d",
                  total_triangles(geoms, num_geoms), h->num_tris);
        return RT_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    std::lock_guard<std::mutex> g(h->mu);
    TmpBuf<float> tmp;
    TmpBuf<int> bad;
    if (!tmp.alloc((size_t)h->num_tris * 9, s) || !bad.alloc(1, s) ||
        !RT_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s)))
        return RT_ERR_NOMEM;
    if (!gather_geometries(geoms, num_geoms, tmp.p, bad.p, s, "cudaBVH_refitGeometries")) return RT_ERR_INVALID;
    if (!RT_CUDA(cudaMemcpyAsync(h->tris9.p, tmp.p, tmp.bytes(), cudaMemcpyDeviceToDevice, s))) return RT_ERR_CUDA;
    return refit_handle(h, s) ? RT_OK : RT_ERR_CUDA;
}

int cudaBVH_serialize(CudaBVH_t h, void* buf, uint64_t capacity, uint64_t* size) {
    clear_error();
    if (!h || !size) {
        set_error("cudaBVH_serialize: invalid argument");
        return RT_ERR_INVALID;
    }
    std::lock_guard<std::mutex> g(h->mu);
    BlobHeader b{};
    memcpy(b.magic, kMagic, 8);
    b.version = kVersion;
    b.header_bytes = sizeof(BlobHeader);
    b.num_tris = h->num_tris;
    b.bvh2_slots = h->bvh2.num_nodes;
    b.num_prims = h->bvh2.num_prims;
    b.num_nodes8 = h->bvh8.num_nodes;
    b.num_items8 = h->bvh8.num_leaf_items;
    b.depth8 = h->bvh8.depth;
    memcpy(b.bmin, h->bmin, sizeof(b.bmin));
    memcpy(b.bmax, h->bmax, sizeof(b.bmax));
    b.stats = h->stats;
    const Sections sec = sections(b);
    b.payload_bytes = sec.total;
    *size = sizeof(BlobHeader) + sec.total;
    if (!buf) return RT_OK;  // size query
    if (capacity < *size) {
        set_error("cudaBVH_serialize: buffer of %llu bytes, %llu needed", (unsigned long long)capacity,
                  (unsigned long long)*size);
        return RT_ERR_CAPACITY;
    }
    unsigned char* p = static_cast<unsigned char*>(buf) + sizeof(BlobHeader);
    memset(p, 0, sec.total);
    size_t o = 0;
    const bool ok =
        RT_CUDA(cudaMemcpy(p + o, h->tris9.p, (size_t)b.num_tris * sizeof(CudaTri), cudaMemcpyDeviceToHost)) &&
        RT_CUDA(cudaMemcpy(p + (o += sec.tris), h->bvh2.nodes.p, (size_t)b.bvh2_slots * sizeof(Node2),
                           cudaMemcpyDeviceToHost)) &&
        RT_CUDA(cudaMemcpy(p + (o += sec.bvh2), h->bvh2.perm.p, (size_t)b.num_prims * sizeof(int),
                           cudaMemcpyDeviceToHost)) &&
        RT_CUDA(cudaMemcpy(p + (o += sec.perm), h->bvh8.nodes.p, (size_t)b.num_nodes8 * sizeof(Bvh8Node),
                           cudaMemcpyDeviceToHost)) &&
        RT_CUDA(cudaMemcpy(p + (o += sec.nodes8), h->bvh8.tris.p, (size_t)b.num_items8 * sizeof(TriRec),
                           cudaMemcpyDeviceToHost));
    if (!ok) return RT_ERR_CUDA;
    b.checksum = checksum(p, sec.total);
    memcpy(buf, &b, sizeof(BlobHeader));
    return RT_OK;
}

CudaBVH_t cudaBVH_deserialize(const void* buf, uint64_t size) {
    clear_error();
    if (!buf || size < sizeof(BlobHeader)) {
        set_error("cudaBVH_deserialize: buffer too small for a header");
        return nullptr;
    }
    BlobHeader b;
    memcpy(&b, buf, sizeof(BlobHeader));
    if (memcmp(b.magic, kMagic, 8) != 0) {
        set_error("cudaBVH_deserialize: not a BVH blob");
        return nullptr;
    }
    if (b.version != kVersion || b.header_bytes != sizeof(BlobHeader)) {
        set_error("cudaBVH_deserialize: blob version %u (header %u bytes); this library reads version %u", b.version,
                  b.header_bytes, kVersion);
        return nullptr;
    }
    if (b.num_tris <= 0 || b.num_prims != b.num_tris || b.bvh2_slots <= 0 || b.bvh2_slots > 2 * b.num_tris ||
        b.num_nodes8 <= 0 || b.num_nodes8 > b.num_tris + 1 || b.num_items8 != b.num_tris || b.depth8 <= 0) {
        set_error("cudaBVH_deserialize: inconsistent counts");
        return nullptr;
    }
    const Sections sec = sections(b);
    if (b.payload_bytes != sec.total || size < sizeof(BlobHeader) + sec.total) {
        set_error("cudaBVH_deserialize: blob truncated (%llu bytes, %llu expected)", (unsigned long long)size,
                  (unsigned long long)(sizeof(BlobHeader) + sec.total));
        return nullptr;
    }
    const unsigned char* p = static_cast<const unsigned char*>(buf) + sizeof(BlobHeader);
    if (checksum(p, sec.total) != b.checksum) {
        set_error("cudaBVH_deserialize: checksum mismatch (corrupted blob)");
        return nullptr;
    }
    if (!check_bvh2(p + sec.tris, b.bvh2_slots, p + sec.tris + sec.bvh2, b.num_prims)) {
        set_error("cudaBVH_deserialize: malformed binary BVH");
        return nullptr;
    }
    CudaBVHHandle* h = create_handle(b.num_tris);
    if (!h) return nullptr;
    size_t o = 0;
    bool ok = h->tris9.alloc((size_t)b.num_tris * 9) && h->bvh2.nodes.alloc((size_t)b.bvh2_slots) &&
              h->bvh2.perm.alloc((size_t)b.num_prims) && h->bvh8.nodes.alloc((size_t)b.num_nodes8) &&
              h->bvh8.tris.alloc((size_t)b.num_items8) &&
              RT_CUDA(cudaMemcpy(h->tris9.p, p + o, (size_t)b.num_tris * sizeof(CudaTri), cudaMemcpyHostToDevice)) &&
              RT_CUDA(cudaMemcpy(h->bvh2.nodes.p, p + (o += sec.tris), (size_t)b.bvh2_slots * sizeof(Node2),
                                 cudaMemcpyHostToDevice)) &&
              RT_CUDA(cudaMemcpy(h->bvh2.perm.p, p + (o += sec.bvh2), (size_t)b.num_prims * sizeof(int),
                                 cudaMemcpyHostToDevice)) &&
              RT_CUDA(cudaMemcpy(h->bvh8.nodes.p, p + (o += sec.perm), (size_t)b.num_nodes8 * sizeof(Bvh8Node),
                                 cudaMemcpyHostToDevice)) &&
              RT_CUDA(cudaMemcpy(h->bvh8.tris.p, p + (o += sec.nodes8), (size_t)b.num_items8 * sizeof(TriRec),
                                 cudaMemcpyHostToDevice)) &&
              ensure_counters(h->counters) && h->status.alloc(1) &&
              RT_CUDA(cudaMemset(h->status.p, 0, sizeof(int)));
    if (ok) {
        h->bvh2.num_nodes = b.bvh2_slots;
        h->bvh2.num_prims = b.num_prims;
        h->bvh2.num_roots = 1;
        h->bvh8.num_nodes = b.num_nodes8;
        h->bvh8.num_leaf_items = b.num_items8;
        h->bvh8.depth = b.depth8;
        memcpy(h->bmin, b.bmin, sizeof(b.bmin));
        memcpy(h->bmax, b.bmax, sizeof(b.bmax));
        for (int a = 0; a < 3; a++) h->center[a] = (b.bmin[a] + b.bmax[a]) * 0.5f;
        const float ex = b.bmax[0] - b.bmin[0], ey = b.bmax[1] - b.bmin[1], ez = b.bmax[2] - b.bmin[2];
        h->extent = sqrtf(ex * ex + ey * ey + ez * ez);
        h->stats = b.stats;
        // the structure is checked before any traversal reads it
        ok = validate_bvh8(h->bvh8, h->bvh8.num_leaf_items, h->num_tris);
    }
    if (!ok) {
        delete h;
        return nullptr;
    }
    return h;
}

}  // extern "C"
