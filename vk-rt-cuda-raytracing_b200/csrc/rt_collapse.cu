// rt_collapse.cu -- BVH2 -> compressed 8-wide nodes (top-down, one thread
// per output node, one launch pair per level).
//
// Which binary nodes become the children of an 8-wide node is decided one
// of two ways.  Greedy: start from the binary node's two children and
// repeatedly open the inner child with the largest surface area until there
// are 8 children or only leaves remain.  SAH-optimal (the dynamic program of
// Ylitie, Karras, Laine, HPG 2017): a bottom-up pass computes, for every
// binary node n and i = 1..8, the least cost of covering n's triangles with
// at most i subtrees (a subtree is an 8-wide node, cost c_node * area, or
// one leaf of at most p_max triangles, cost c_prim * area * count), and the
// top-down pass expands every 8-wide node's children along the recorded
// choices; small subtrees can thus become one leaf and nodes come out
// fuller.  Either way: assign the children to octant slots
// (slot s takes the child nearest along the direction with sign bits s,
// greedy on the projected-centroid cost); quantise each child box to 8 bits
// per plane, rounded outward, on the grid p + q * 2^e; write the triangle
// records of the leaf children contiguously in slot order.
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <vector>

#include <cuda/atomic>

#include "rt_internal.h"

namespace rtb {

struct Gather {
    int kid[8];  // binary node id per slot, -1 = empty
};

// Per binary node, for the SAH-optimal collapse.
struct DPNode {
    float c[8];          // c[i]: least cost of covering the subtree with at most i + 1 subtrees
    unsigned char d[8];  // d[0]: 1 if the subtree is best one leaf; d[i], i >= 1: split k for c[i], 0 = as c[i-1]
    unsigned char s8;    // split of the 8 slots between the children when the node is an 8-wide node
    unsigned char pad[3];
    int first, count;    // triangle range in the permutation (first -1: not contiguous)
};

__device__ __forceinline__ float node_area(const Node2& n) {
    const float dx = n.hi[0] - n.lo[0], dy = n.hi[1] - n.lo[1], dz = n.hi[2] - n.lo[2];
    return dx * dy + dy * dz + dz * dx;
}
__device__ __forceinline__ bool is_leaf2(const Node2& n) { return n.b < 0; }

__global__ void k_dp_parents(const Node2* __restrict__ nodes, int slots, int* __restrict__ parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= slots) return;
    const Node2 nd = nodes[i];
    if (nd.b > 0) {  // inner node (unused reserved slots have b == 0)
        parent[nd.a] = i;
        parent[nd.b] = i;
    }
}

// Bottom-up: one thread per binary leaf walks toward its root; at every node
// the second child to arrive fills the node's table (an acquire-release
// arrival counter, L2 loads after it).  Depth is bounded by the builder.
__global__ void k_dp(const Node2* __restrict__ nodes, int slots, const int* __restrict__ parent,
                     int* __restrict__ arrive, DPNode* __restrict__ dp, float c_node, float c_prim, int p_max,
                     int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= slots) return;
    const Node2 lf = nodes[i];
    if (lf.b >= 0) return;  // leaves only
    {
        DPNode t;
        const float v = c_prim * node_area(lf) * (float)(-lf.b);
        for (int k = 0; k < 8; k++) {
            t.c[k] = v;
            t.d[k] = 0;
        }
        t.d[0] = 1;
        t.s8 = 0;
        t.first = lf.a;
        t.count = -lf.b;
        dp[i] = t;
    }
    int cur = i;
    for (int step = 0;; step++) {
        const int par = parent[cur];
        if (par < 0) return;
        if (step >= 256) {  // deeper than any tree the builder makes: give up (greedy collapse instead)
            atomicOr(status, 1);
            return;
        }
        // release our table, acquire the sibling's: the second arrival sees
        // both (measured 4.66 -> 3.99 ms over two full fences on 22M triangles)
        cuda::atomic_ref<int, cuda::thread_scope_device> arr(arrive[par]);
        if (arr.fetch_add(1, cuda::memory_order_acq_rel) == 0) return;
        const Node2 n = nodes[par];
        float cl[8], cr[8];
        for (int k = 0; k < 8; k++) {
            cl[k] = __ldcg(&dp[n.a].c[k]);
            cr[k] = __ldcg(&dp[n.b].c[k]);
        }
        const int fl = __ldcg(&dp[n.a].first), nl = __ldcg(&dp[n.a].count);
        const int fr = __ldcg(&dp[n.b].first), nr = __ldcg(&dp[n.b].count);
        DPNode t;
        t.count = nl + nr;
        t.first = (fl >= 0 && fr >= 0 && (fl + nl == fr || fr + nr == fl)) ? min(fl, fr) : -1;
        float D[9];
        unsigned char K[9];
        for (int j = 2; j <= 8; j++) {
            float best = INFINITY;
            unsigned char bk = 1;
            for (int k = 1; k < j; k++) {
                const float v = cl[k - 1] + cr[j - k - 1];
                if (v < best) { best = v; bk = (unsigned char)k; }
            }
            D[j] = best;
            K[j] = bk;
        }
        const float a = node_area(n);
        const float c_int = c_node * a + D[8];
        const float c_leaf = (t.first >= 0 && t.count <= p_max) ? c_prim * a * (float)t.count : INFINITY;
        t.c[0] = fminf(c_int, c_leaf);
        t.d[0] = c_leaf <= c_int ? 1 : 0;
        t.s8 = K[8];
        for (int k = 1; k < 8; k++) {
            if (D[k + 1] < t.c[k - 1]) {
                t.c[k] = D[k + 1];
                t.d[k] = K[k + 1];
            } else {
                t.c[k] = t.c[k - 1];
                t.d[k] = 0;
            }
        }
        dp[par] = t;
        cur = par;
    }
}

__device__ void gather_dp_one(int i, const Node2* __restrict__ nodes, const DPNode* __restrict__ dp,
                              const int* __restrict__ level, Gather* __restrict__ out, int* __restrict__ n_inner,
                              int* __restrict__ n_items) {
    const int b2 = level[i];
    const Node2 me = nodes[b2];
    int kid[8];
    int nk = 0;
    if (is_leaf2(me)) {
        kid[nk++] = b2;
    } else {
        // expand the two children under the 8-slot budget along the recorded splits
        int sx[16], sj[16], sp = 0;
        const int k8 = dp[b2].s8;
        sx[sp] = me.b; sj[sp++] = 8 - k8;
        sx[sp] = me.a; sj[sp++] = k8;
        while (sp > 0 && nk < 8) {
            const int x = sx[--sp];
            int j = sj[sp];
            while (j > 1 && dp[x].d[j - 1] == 0) j--;
            if (j == 1 || sp > 13) {
                kid[nk++] = x;
            } else {
                const int k = dp[x].d[j - 1];
                const Node2 c = nodes[x];
                sx[sp] = c.b; sj[sp++] = j - k;
                sx[sp] = c.a; sj[sp++] = k;
            }
        }
    }
    // octant slot assignment
    float pc[3];
    for (int a = 0; a < 3; a++) pc[a] = (me.lo[a] + me.hi[a]) * 0.5f;
    float cost[8][8];
    for (int k = 0; k < nk; k++) {
        const Node2 c = nodes[kid[k]];
        float d[3];
        for (int a = 0; a < 3; a++) d[a] = (c.lo[a] + c.hi[a]) * 0.5f - pc[a];
        for (int s = 0; s < 8; s++)
            cost[k][s] = ((s & 1) ? -d[0] : d[0]) + ((s & 2) ? -d[1] : d[1]) + ((s & 4) ? -d[2] : d[2]);
    }
    int slot_kid[8];
    for (int s = 0; s < 8; s++) slot_kid[s] = -1;
    unsigned used_k = 0, used_s = 0;
    for (int r = 0; r < nk; r++) {
        float bc = FLT_MAX;
        int bk = -1, bs = -1;
        for (int k = 0; k < nk; k++) {
            if (used_k & (1u << k)) continue;
            for (int s = 0; s < 8; s++) {
                if (used_s & (1u << s)) continue;
                if (cost[k][s] < bc || bk < 0) { bc = cost[k][s]; bk = k; bs = s; }
            }
        }
        used_k |= 1u << bk;
        used_s |= 1u << bs;
        slot_kid[bs] = kid[bk];
    }
    Gather g;
    int ni = 0, nt = 0;
    for (int s = 0; s < 8; s++) {
        g.kid[s] = slot_kid[s];
        if (slot_kid[s] < 0) continue;
        const int x = slot_kid[s];
        if (is_leaf2(nodes[x]) || dp[x].d[0]) nt += dp[x].count;
        else ni++;
    }
    out[i] = g;
    n_inner[i] = ni;
    n_items[i] = nt;
}

__device__ void gather_greedy_one(int i, const Node2* __restrict__ nodes, const int* __restrict__ level,
                                  Gather* __restrict__ out, int* __restrict__ n_inner, int* __restrict__ n_items) {
    const int b2 = level[i];
    const Node2 me = nodes[b2];
    int kid[8];
    int nk = 0;
    if (is_leaf2(me)) {
        kid[nk++] = b2;
    } else {
        kid[nk++] = me.a;
        kid[nk++] = me.b;
        while (nk < 8) {
            int best = -1;
            float ba = -1.f;
            for (int k = 0; k < nk; k++) {
                const Node2 c = nodes[kid[k]];
                if (!is_leaf2(c)) {
                    const float a = node_area(c);
                    if (a > ba) { ba = a; best = k; }
                }
            }
            if (best < 0) break;
            const Node2 c = nodes[kid[best]];
            kid[best] = c.a;
            kid[nk++] = c.b;
        }
    }
    // octant slot assignment
    float pc[3];
    for (int a = 0; a < 3; a++) pc[a] = (me.lo[a] + me.hi[a]) * 0.5f;
    float cost[8][8];
    for (int k = 0; k < nk; k++) {
        const Node2 c = nodes[kid[k]];
        float d[3];
        for (int a = 0; a < 3; a++) d[a] = (c.lo[a] + c.hi[a]) * 0.5f - pc[a];
        for (int s = 0; s < 8; s++)
            cost[k][s] = ((s & 1) ? -d[0] : d[0]) + ((s & 2) ? -d[1] : d[1]) + ((s & 4) ? -d[2] : d[2]);
    }
    int slot_kid[8];
    for (int s = 0; s < 8; s++) slot_kid[s] = -1;
    unsigned used_k = 0, used_s = 0;
    for (int r = 0; r < nk; r++) {
        float bc = FLT_MAX;
        int bk = -1, bs = -1;
        for (int k = 0; k < nk; k++) {
            if (used_k & (1u << k)) continue;
            for (int s = 0; s < 8; s++) {
                if (used_s & (1u << s)) continue;
                if (cost[k][s] < bc || bk < 0) { bc = cost[k][s]; bk = k; bs = s; }
            }
        }
        used_k |= 1u << bk;
        used_s |= 1u << bs;
        slot_kid[bs] = kid[bk];
    }
    Gather g;
    int ni = 0, nt = 0;
    for (int s = 0; s < 8; s++) {
        g.kid[s] = slot_kid[s];
        if (slot_kid[s] < 0) continue;
        const Node2 c = nodes[slot_kid[s]];
        if (is_leaf2(c)) nt += -c.b;
        else ni++;
    }
    out[i] = g;
    n_inner[i] = ni;
    n_items[i] = nt;
}

// The collapse's level loop keeps its state on the device, so a level can
// be enqueued without the host knowing its width (the graph-driven build
// runs the loop under a conditional node; the host-driven loop reads the
// totals only to decide when to stop).
// More 8-wide levels than any tree the builder makes (its binary depth is
// bounded); the graph-driven loop stops there with status 2.
constexpr int kMaxCollapseLevels = 1024;
struct CollapseLevel {
    int L;           // binary nodes turned into 8-wide nodes at this level
    int level_base;  // first 8-wide node of this level
    int items;       // leaf items (triangle records / instance slots) written so far
    int depth;       // levels done
    int status;      // 1: node or item capacity exceeded; 2: too many levels
    int pad[3];
};

// The DP tables are used unless the bottom-up pass gave up (too deep).
__device__ __forceinline__ const DPNode* dp_in_use(const DPNode* dp, const int* dp_status) {
    return dp && dp_status && *dp_status == 0 ? dp : nullptr;
}

// One thread per binary node of the level (grid-stride over lv->L).
__global__ void k_gather_lv(const Node2* __restrict__ nodes, const DPNode* __restrict__ dp,
                            const int* __restrict__ dp_status, const int* __restrict__ level,
                            const CollapseLevel* __restrict__ lv, Gather* __restrict__ out,
                            int* __restrict__ n_inner, int* __restrict__ n_items) {
    const int L = lv->L;
    const DPNode* d = dp_in_use(dp, dp_status);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L; i += gridDim.x * blockDim.x) {
        if (d) gather_dp_one(i, nodes, d, level, out, n_inner, n_items);
        else gather_greedy_one(i, nodes, level, out, n_inner, n_items);
    }
}

// smallest e with 255 * 2^e >= ext (ext > 0), from the exact double value
__device__ __forceinline__ int grid_exponent(double ext) {
    int k;
    const double m = frexp(ext / 255.0, &k);  // ext/255 = m * 2^k, m in [0.5, 1)
    int e = (m == 0.5) ? k - 1 : k;
    // ext/255 rounding in double can undershoot by one ulp; make sure 255*2^e >= ext
    if (ldexp(255.0, e) < ext) e++;
    return e;
}

__device__ void emit_one(int i, const Node2* __restrict__ nodes, const Gather* __restrict__ gat,
                         const int* __restrict__ inner_off, const int* __restrict__ item_off, int child_base0,
                         int item_base0, const int* __restrict__ perm, const float* __restrict__ tris9,
                         Bvh8Node* __restrict__ out_nodes, int out_base, TriRec* __restrict__ out_tris,
                         int* __restrict__ out_ids, int* __restrict__ next_level, const DPNode* __restrict__ dp) {
    const Gather g = gat[i];
    const int child_base = child_base0 + inner_off[i];
    const int tri_base = item_base0 + item_off[i];
    // node box = union of the children
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int s = 0; s < 8; s++) {
        if (g.kid[s] < 0) continue;
        const Node2 c = nodes[g.kid[s]];
        for (int a = 0; a < 3; a++) {
            lo[a] = fminf(lo[a], c.lo[a]);
            hi[a] = fmaxf(hi[a], c.hi[a]);
        }
    }
    uint32_t ebytes[3];
    double scale[3];
    for (int a = 0; a < 3; a++) {
        const double ext = (double)hi[a] - (double)lo[a];
        if (!(ext > 0.0)) {
            ebytes[a] = 0;
            scale[a] = 0.0;
        } else {
            int e = grid_exponent(ext);
            if (e < -126) e = -126;
            if (e > 127) e = 127;
            ebytes[a] = (uint32_t)(e + 127);
            scale[a] = ldexp(1.0, e);
        }
    }
    uint32_t imask = 0;
    uint32_t meta[2] = {0, 0};
    uint32_t qlo[3][2] = {{0, 0}, {0, 0}, {0, 0}}, qhi[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    int inner_seen = 0, offset = 0;
    for (int s = 0; s < 8; s++) {
        const int k = g.kid[s];
        if (k < 0) continue;
        const Node2 c = nodes[k];
        for (int a = 0; a < 3; a++) {
            uint32_t ql = 0, qh = 0;
            if (scale[a] > 0.0) {
                double fl = floor(((double)c.lo[a] - (double)lo[a]) / scale[a]);
                double ch = ceil(((double)c.hi[a] - (double)lo[a]) / scale[a]);
                fl = fmin(fmax(fl, 0.0), 255.0);
                ch = fmin(fmax(ch, 0.0), 255.0);
                ql = (uint32_t)fl;
                qh = (uint32_t)ch;
            }
            qlo[a][s >> 2] |= ql << ((s & 3) * 8);
            qhi[a][s >> 2] |= qh << ((s & 3) * 8);
        }
        uint32_t m;
        // a leaf child is a binary leaf, or with the SAH-optimal collapse a
        // subtree chosen to be one leaf (its triangles are contiguous)
        const bool as_leaf = is_leaf2(c) || (dp && dp[k].d[0]);
        if (as_leaf) {
            const int cnt = dp ? dp[k].count : -c.b;
            const int first = dp ? dp[k].first : c.a;
            m = ((uint32_t)cnt << 5) | (uint32_t)offset;
            for (int j = 0; j < cnt; j++) {
                const int prim = perm[first + j];
                const int dst = tri_base + offset + j;
                if (tris9) {
                    const float* t = tris9 + (size_t)prim * 9;
                    TriRec r;
                    r.a = make_float4(t[0], t[1], t[2], __int_as_float(prim));
                    r.b = make_float4(__fsub_rn(t[3], t[0]), __fsub_rn(t[4], t[1]), __fsub_rn(t[5], t[2]), 0.f);
                    r.c = make_float4(__fsub_rn(t[6], t[0]), __fsub_rn(t[7], t[1]), __fsub_rn(t[8], t[2]), 0.f);
                    out_tris[dst] = r;
                } else {
                    out_ids[dst] = prim;
                }
            }
            offset += cnt;
        } else {
            imask |= 1u << s;
            m = 0xFFu;
            next_level[inner_off[i] + inner_seen] = k;
            inner_seen++;
        }
        meta[s >> 2] |= m << ((s & 3) * 8);
    }
    Bvh8Node nd;
    nd.w[0] = make_uint4(__float_as_uint(lo[0]), __float_as_uint(lo[1]), __float_as_uint(lo[2]),
                         ebytes[0] | (ebytes[1] << 8) | (ebytes[2] << 16) | (imask << 24));
    nd.w[1] = make_uint4((uint32_t)child_base, (uint32_t)tri_base, meta[0], meta[1]);
    nd.w[2] = make_uint4(qlo[0][0], qlo[0][1], qhi[0][0], qhi[0][1]);
    nd.w[3] = make_uint4(qlo[1][0], qlo[1][1], qhi[1][0], qhi[1][1]);
    nd.w[4] = make_uint4(qlo[2][0], qlo[2][1], qhi[2][0], qhi[2][1]);
    out_nodes[out_base + i] = nd;
}

// One thread per binary node of the level (grid-stride over lv->L): this
// level's 8-wide nodes go to lv->level_base + i, their inner children to
// the next level's list, their leaves' records after lv->items.
// Writes nothing when the level's totals (tot: inner children, leaf items)
// would pass the capacities; k_collapse_advance then reports it.
__global__ void k_emit_lv(const Node2* __restrict__ nodes, const CollapseLevel* __restrict__ lv,
                          const Gather* __restrict__ gat, const int* __restrict__ inner_off,
                          const int* __restrict__ item_off, const int* __restrict__ tot, int max_nodes, int max_items,
                          const int* __restrict__ perm, const float* __restrict__ tris9,
                          Bvh8Node* __restrict__ out_nodes, TriRec* __restrict__ out_tris, int* __restrict__ out_ids,
                          int* __restrict__ next_level, const DPNode* __restrict__ dp,
                          const int* __restrict__ dp_status) {
    const int L = lv->L, base = lv->level_base, items = lv->items;
    if (base + L + tot[0] > max_nodes || items + tot[1] > max_items) return;
    const DPNode* d = dp_in_use(dp, dp_status);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L; i += gridDim.x * blockDim.x)
        emit_one(i, nodes, gat, inner_off, item_off, base + L, items, perm, tris9, out_nodes, base, out_tris, out_ids,
                 next_level, d);
}

// Level 0: the roots (binary nodes 0 .. R-1 -> 8-wide nodes 0 .. R-1).
template <bool COND>
__global__ void k_collapse_init(CollapseLevel* __restrict__ lv, int* __restrict__ level, int R,
                                cudaGraphConditionalHandle cond) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < R; i += gridDim.x * blockDim.x) level[i] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        CollapseLevel z = {};
        z.L = R;
        *lv = z;
        if (COND) cudaGraphSetConditional(cond, R > 0 ? 1u : 0u);
    }
}

// End of a level: tot = {inner children, leaf items} of the level.  Checks
// the capacities, advances the level record, and (graph-driven) continues
// the loop while the next level has nodes and nothing overflowed.
template <bool COND>
__global__ void k_collapse_advance(CollapseLevel* __restrict__ lv, const int* __restrict__ tot, int max_nodes,
                                   int max_items, cudaGraphConditionalHandle cond) {
    CollapseLevel v = *lv;
    const int child_base = v.level_base + v.L;
    if (child_base + tot[0] > max_nodes || v.items + tot[1] > max_items) v.status |= 1;
    if (v.depth + 1 >= kMaxCollapseLevels && tot[0] > 0) v.status |= 2;  // bounds the graph's loop
    v.level_base = child_base;
    v.items += tot[1];
    v.L = v.status ? 0 : tot[0];
    v.depth++;
    *lv = v;
    if (COND) cudaGraphSetConditional(cond, v.L > 0 ? 1u : 0u);
}

// Next level's node list becomes the current one (graph-driven loop, whose
// kernels keep fixed buffer arguments).
__global__ void k_copy_level(const int* __restrict__ src, int* __restrict__ dst, const CollapseLevel* __restrict__ lv) {
    const int L = lv->L;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

// The level record's totals for the host: {nodes, leaf items, depth, status}.
__global__ void k_collapse_result(const CollapseLevel* __restrict__ lv, int* __restrict__ out) {
    out[0] = lv->level_base;
    out[1] = lv->items;
    out[2] = lv->depth;
    out[3] = lv->status;
}

namespace {
// SAH-optimal collapse for triangle BLASes unless RTB200_COLLAPSE=greedy
// (TLAS leaves stay single instances: greedy); its cost constants.
int collapse_mode() {
    static const int mode = [] {
        const char* e = getenv("RTB200_COLLAPSE");
        return e && !strcmp(e, "greedy") ? 0 : 1;
    }();
    return mode;
}
float dp_c_prim() {
    static const float c = [] {
        const char* e = getenv("RTB200_DP_CPRIM");
        return e ? (float)atof(e) : 0.5f;
    }();
    return c;
}
int dp_p_max() {
    static const int p = [] {
        const char* e = getenv("RTB200_DP_PMAX");
        const int v = e ? atoi(e) : 4;
        return v < 1 ? 1 : (v > 4 ? 4 : v);
    }();
    return p;
}
}  // namespace

bool collapse_bvh8(const Bvh2Device& b2, const float* d_tris9, Bvh8Device& out, cudaStream_t s) {
    const int n = b2.num_prims;
    const int R = b2.num_roots;
    // upper bound on 8-wide nodes: every node has >= 2 children except a
    // root that is a single leaf, so nodes <= leaves + roots <= n + R
    const int max_nodes = n + R;
    // the output: a caller's buffers when large enough, else allocated here
    if (!out.nodes.ensure(max_nodes)) return false;
    if (d_tris9) {
        if (!out.tris.ensure(n)) return false;
    } else {
        if (!out.leaf_ids.ensure(n)) return false;
    }
    TmpBuf<int> lvl_a, lvl_b, n_inner, n_items, inner_off, item_off, tot;
    TmpBuf<Gather> gat;
    TmpBuf<CollapseLevel> lv;
    if (!lvl_a.alloc(max_nodes, s) || !lvl_b.alloc(max_nodes, s) || !n_inner.alloc(max_nodes, s) ||
        !n_items.alloc(max_nodes, s) || !inner_off.alloc(max_nodes, s) || !item_off.alloc(max_nodes, s) ||
        !gat.alloc(max_nodes, s) || !tot.alloc(2, s) || !lv.alloc(1, s))
        return false;
    TmpBuf<DPNode> dp;
    TmpBuf<int> parent, arrive, st;  // st: 1 when the bottom-up pass gave up (greedy collapse instead)
    if (d_tris9 && collapse_mode() == 1) {
        const int slots = b2.num_nodes;
        if (!dp.alloc(slots, s) || !parent.alloc(slots, s) || !arrive.alloc(slots, s) || !st.alloc(1, s)) return false;
        if (!RT_CUDA(cudaMemsetAsync(parent.p, 0xFF, sizeof(int) * (size_t)slots, s)) ||
            !RT_CUDA(cudaMemsetAsync(arrive.p, 0, sizeof(int) * (size_t)slots, s)) ||
            !RT_CUDA(cudaMemsetAsync(st.p, 0, sizeof(int), s)))
            return false;
        k_dp_parents<<<(slots + 255) / 256, 256, 0, s>>>(b2.nodes.p, slots, parent.p);
        k_dp<<<(slots + 255) / 256, 256, 0, s>>>(b2.nodes.p, slots, parent.p, arrive.p, dp.p, 1.0f, dp_c_prim(),
                                                 dp_p_max(), st.p);
    }
    int* cur = lvl_a.p;
    int* nxt = lvl_b.p;
    k_collapse_init<false><<<(R + 255) / 256, 256, 0, s>>>(lv.p, cur, R, 0);
    int L = R, level_base = 0, items = 0, depth = 0;
    while (L > 0) {
        const int grid = (L + 127) / 128;
        k_gather_lv<<<grid, 128, 0, s>>>(b2.nodes.p, dp.p, st.p, cur, lv.p, gat.p, n_inner.p, n_items.p);
        if (!scan_exclusive(n_inner.p, inner_off.p, L, tot.p, s)) return false;
        if (!scan_exclusive(n_items.p, item_off.p, L, tot.p + 1, s)) return false;
        int h[2];
        cudaMemcpyAsync(h, tot.p, sizeof(h), cudaMemcpyDeviceToHost, s);
        if (!RT_CUDA(cudaStreamSynchronize(s))) return false;
        const int child_base = level_base + L;
        if (child_base + h[0] > max_nodes || items + h[1] > n) {
            set_error("collapse: capacity exceeded");
            return false;
        }
        k_emit_lv<<<grid, 128, 0, s>>>(b2.nodes.p, lv.p, gat.p, inner_off.p, item_off.p, tot.p, max_nodes, n,
                                       b2.perm.p, d_tris9, out.nodes.p, out.tris.p, out.leaf_ids.p, nxt, dp.p, st.p);
        k_collapse_advance<false><<<1, 1, 0, s>>>(lv.p, tot.p, max_nodes, n, 0);
        level_base = child_base;
        items += h[1];
        L = h[0];
        std::swap(cur, nxt);
        depth++;
    }
    out.num_nodes = level_base;
    out.num_leaf_items = items;
    out.depth = depth;
    return RT_CUDA(cudaGetLastError());
}

size_t collapse_graph_scratch_bytes(int n, int R, int slots, bool dp) {
    const size_t max_nodes = (size_t)n + R;
    size_t b = max_nodes * (6 * sizeof(int) + sizeof(Gather)) + 2 * sizeof(int) + sizeof(CollapseLevel) +
               2 * scan_scratch_ints((int)max_nodes) * sizeof(int) + 16 * 256;
    if (dp) b += (size_t)slots * (sizeof(DPNode) + 2 * sizeof(int)) + sizeof(int);
    return b;
}

bool enqueue_collapse_graph(const Node2* nodes2, const int* perm, int n, int R, int slots, const float* d_tris9,
                            Bvh8Node* out_nodes, TriRec* out_tris, int* out_ids, char* scratch, size_t scratch_bytes,
                            int* d_result, cudaStream_t cs, cudaStream_t bs) {
    const int max_nodes = n + R;
    const bool use_dp = d_tris9 && collapse_mode() == 1;
    if (collapse_graph_scratch_bytes(n, R, slots, use_dp) > scratch_bytes) {
        set_error("collapse: graph scratch too small");
        return false;
    }
    char* q = scratch;
    auto take = [&q](size_t bytes) {
        char* r = q;
        q += (bytes + 255) & ~size_t(255);
        return r;
    };
    const size_t scan_ints = scan_scratch_ints(max_nodes);
    int* lvl_a = reinterpret_cast<int*>(take(sizeof(int) * (size_t)max_nodes));
    int* lvl_b = reinterpret_cast<int*>(take(sizeof(int) * (size_t)max_nodes));
    int* n_inner = reinterpret_cast<int*>(take(sizeof(int) * (size_t)max_nodes));
    int* n_items = reinterpret_cast<int*>(take(sizeof(int) * (size_t)max_nodes));
    int* inner_off = reinterpret_cast<int*>(take(sizeof(int) * (size_t)max_nodes));
    int* item_off = reinterpret_cast<int*>(take(sizeof(int) * (size_t)max_nodes));
    Gather* gat = reinterpret_cast<Gather*>(take(sizeof(Gather) * (size_t)max_nodes));
    int* tot = reinterpret_cast<int*>(take(2 * sizeof(int)));
    CollapseLevel* lv = reinterpret_cast<CollapseLevel*>(take(sizeof(CollapseLevel)));
    int* scan_a = reinterpret_cast<int*>(take(sizeof(int) * scan_ints));
    int* scan_b = reinterpret_cast<int*>(take(sizeof(int) * scan_ints));
    DPNode* dp = nullptr;
    int *parent = nullptr, *arrive = nullptr, *st = nullptr;
    if (use_dp) {
        dp = reinterpret_cast<DPNode*>(take(sizeof(DPNode) * (size_t)slots));
        parent = reinterpret_cast<int*>(take(sizeof(int) * (size_t)slots));
        arrive = reinterpret_cast<int*>(take(sizeof(int) * (size_t)slots));
        st = reinterpret_cast<int*>(take(sizeof(int)));
        if (!RT_CUDA(cudaMemsetAsync(parent, 0xFF, sizeof(int) * (size_t)slots, cs)) ||
            !RT_CUDA(cudaMemsetAsync(arrive, 0, sizeof(int) * (size_t)slots, cs)) ||
            !RT_CUDA(cudaMemsetAsync(st, 0, sizeof(int), cs)))
            return false;
        k_dp_parents<<<(slots + 255) / 256, 256, 0, cs>>>(nodes2, slots, parent);
        k_dp<<<(slots + 255) / 256, 256, 0, cs>>>(nodes2, slots, parent, arrive, dp, 1.0f, dp_c_prim(), dp_p_max(),
                                                  st);
    }
    cudaGraphConditionalHandle cond;
    cudaGraph_t body;
    if (!capture_conditional_handle(cs, &cond)) return false;
    k_collapse_init<true><<<(R + 255) / 256, 256, 0, cs>>>(lv, lvl_a, R, cond);
    if (!capture_while(cs, cond, &body)) return false;
    if (!RT_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)))
        return false;
    // grid-stride kernels: a level is at most max_nodes wide
    const int grid = std::max(1, std::min((max_nodes + 127) / 128, num_sms() * 16));
    k_gather_lv<<<grid, 128, 0, bs>>>(nodes2, dp, st, lvl_a, lv, gat, n_inner, n_items);
    bool ok = scan_exclusive_dev(n_inner, inner_off, max_nodes, &lv->L, tot, scan_a, bs) &&
              scan_exclusive_dev(n_items, item_off, max_nodes, &lv->L, tot + 1, scan_b, bs);
    if (ok) {
        k_emit_lv<<<grid, 128, 0, bs>>>(nodes2, lv, gat, inner_off, item_off, tot, max_nodes, n, perm, d_tris9,
                                        out_nodes, out_tris, out_ids, lvl_b, dp, st);
        k_collapse_advance<true><<<1, 1, 0, bs>>>(lv, tot, max_nodes, n, cond);
        k_copy_level<<<grid, 128, 0, bs>>>(lvl_b, lvl_a, lv);
        ok = RT_CUDA(cudaGetLastError());
    }
    cudaGraph_t done = nullptr;
    const bool ended = RT_CUDA(cudaStreamEndCapture(bs, &done));
    if (!ok || !ended) return false;
    // results for the host: nodes, leaf items, depth, status
    k_collapse_result<<<1, 1, 0, cs>>>(lv, d_result);
    return RT_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- SAH --
__global__ void k_sah(const Node2* __restrict__ nodes, int m, float* __restrict__ acc) {
    float s = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const Node2 n = nodes[i];
        if (n.b == 0 && i != 0) continue;  // unused reserved slot
        const float dx = n.hi[0] - n.lo[0], dy = n.hi[1] - n.lo[1], dz = n.hi[2] - n.lo[2];
        const float a = dx * dy + dy * dz + dz * dx;
        s += n.b < 0 ? a * (float)(-n.b) : a;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc, s);
}

float bvh2_sah_cost(const Bvh2Device& b2, cudaStream_t s) {
    TmpBuf<float> acc;
    if (!acc.alloc(1, s)) return -1.f;
    cudaMemsetAsync(acc.p, 0, sizeof(float), s);
    k_sah<<<std::min((b2.num_nodes + 255) / 256, 1024), 256, 0, s>>>(b2.nodes.p, b2.num_nodes, acc.p);
    float total = 0.f;
    Node2 root;
    cudaMemcpyAsync(&total, acc.p, sizeof(float), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&root, b2.nodes.p, sizeof(Node2), cudaMemcpyDeviceToHost, s);
    if (!RT_CUDA(cudaStreamSynchronize(s))) return -1.f;
    const float dx = root.hi[0] - root.lo[0], dy = root.hi[1] - root.lo[1], dz = root.hi[2] - root.lo[2];
    const float ra = dx * dy + dy * dz + dz * dx;
    return ra > 0.f ? total / ra : 0.f;
}

}  // namespace rtb
