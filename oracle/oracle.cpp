// oracle.cpp -- CPU oracle (TEST INFRASTRUCTURE ONLY; see oracle.h).
//
// Compiled with -ffp-contract=off so every float expression rounds exactly as
// written; the CUDA kernels spell the same intersection arithmetic with
// explicit round-to-nearest intrinsics, which makes hit ids and t bit-exact.
#include "oracle.h"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <thread>
#include <vector>

namespace {

struct V3 { float x, y, z; };
struct Tri { V3 v0, v1, v2; };
struct Box { V3 mn, mx; };

// triAABB / mergeAABB / saArea: layer/cuda_bvh_backend.cu:186-197
Box tri_box(const Tri& t) {
    return {{fminf(fminf(t.v0.x, t.v1.x), t.v2.x), fminf(fminf(t.v0.y, t.v1.y), t.v2.y),
             fminf(fminf(t.v0.z, t.v1.z), t.v2.z)},
            {fmaxf(fmaxf(t.v0.x, t.v1.x), t.v2.x), fmaxf(fmaxf(t.v0.y, t.v1.y), t.v2.y),
             fmaxf(fmaxf(t.v0.z, t.v1.z), t.v2.z)}};
}
Box merge(const Box& a, const Box& b) {
    return {{fminf(a.mn.x, b.mn.x), fminf(a.mn.y, b.mn.y), fminf(a.mn.z, b.mn.z)},
            {fmaxf(a.mx.x, b.mx.x), fmaxf(a.mx.y, b.mx.y), fmaxf(a.mx.z, b.mx.z)}};
}
float area(const Box& b) {
    float dx = b.mx.x - b.mn.x, dy = b.mx.y - b.mn.y, dz = b.mx.z - b.mn.z;
    return 2.f * (dx * dy + dy * dz + dz * dx);
}
inline float axis(const V3& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

struct Node2 { Box box; int left, right, tri_start, tri_count; };

// Binned-SAH BVH2: layer/cuda_bvh_backend.cu:201-251 (NB=16, leaf<=3) and
// cuda_rt_v40.cu:790-840 (NB=32, maxLeaf).  Same split search, same sort,
// same fallbacks, so the output is byte-identical to the reference's.
struct Builder {
    int nbins = 16, max_leaf = 3;
    std::vector<Node2> nodes;
    std::vector<Tri> ordered;
    std::vector<int> orig;
    std::vector<Box> pbox;
    std::vector<V3> cent;
    const Tri* src = nullptr;

    void build(const Tri* t, int n) {
        src = t;
        pbox.resize(n);
        cent.resize(n);
        nodes.reserve((size_t)n * 2);
        for (int i = 0; i < n; i++) {
            pbox[i] = tri_box(t[i]);
            cent[i] = {(pbox[i].mn.x + pbox[i].mx.x) * .5f, (pbox[i].mn.y + pbox[i].mx.y) * .5f,
                       (pbox[i].mn.z + pbox[i].mx.z) * .5f};
        }
        std::vector<int> idx(n);
        for (int i = 0; i < n; i++) idx[i] = i;
        if (n > 0) rec(idx, 0, n);
    }

    int rec(std::vector<int>& idx, int s, int e) {
        Node2 nd;
        nd.tri_start = nd.tri_count = nd.left = nd.right = 0;
        nd.box = pbox[idx[s]];
        for (int i = s + 1; i < e; i++) nd.box = merge(nd.box, pbox[idx[i]]);
        int cnt = e - s;
        if (cnt <= max_leaf) {
            nd.tri_start = (int)ordered.size();
            nd.tri_count = cnt;
            for (int i = s; i < e; i++) { ordered.push_back(src[idx[i]]); orig.push_back(idx[i]); }
            nodes.push_back(nd);
            return (int)nodes.size() - 1;
        }
        const int NB = nbins;
        float best_cost = 1e30f;
        int best_axis = 0, best_split = s + cnt / 2;
        float pA = area(nd.box);
        std::vector<Box> lb(NB), rb(NB);
        std::vector<int> lc(NB), rc(NB);
        for (int ax = 0; ax < 3; ax++) {
            float cmin = 1e30f, cmax = -1e30f;
            for (int i = s; i < e; i++) {
                float c = axis(cent[idx[i]], ax);
                cmin = fminf(cmin, c);
                cmax = fmaxf(cmax, c);
            }
            if (cmax - cmin < 1e-8f) continue;
            for (int b = 0; b < NB; b++) {
                lb[b].mn = {1e30f, 1e30f, 1e30f}; lb[b].mx = {-1e30f, -1e30f, -1e30f}; lc[b] = 0;
                rb[b].mn = {1e30f, 1e30f, 1e30f}; rb[b].mx = {-1e30f, -1e30f, -1e30f}; rc[b] = 0;
            }
            for (int i = s; i < e; i++) {
                float c = axis(cent[idx[i]], ax);
                int b = (int)((c - cmin) / (cmax - cmin) * (NB - 1));
                b = b < 0 ? 0 : (b >= NB ? NB - 1 : b);
                lb[b] = (lc[b] == 0) ? pbox[idx[i]] : merge(lb[b], pbox[idx[i]]);
                lc[b]++;
            }
            for (int b = 1; b < NB; b++) {
                if (lc[b] && lc[b - 1]) lb[b] = merge(lb[b], lb[b - 1]);
                else if (lc[b - 1]) lb[b] = lb[b - 1];
                lc[b] += lc[b - 1];
            }
            for (int i = e - 1; i >= s; i--) {
                float c = axis(cent[idx[i]], ax);
                int b = (int)((c - cmin) / (cmax - cmin) * (NB - 1));
                b = b < 0 ? 0 : (b >= NB ? NB - 1 : b);
                rb[b] = (rc[b] == 0) ? pbox[idx[i]] : merge(rb[b], pbox[idx[i]]);
                rc[b]++;
            }
            for (int b = NB - 2; b >= 0; b--) {
                if (rc[b] && rc[b + 1]) rb[b] = merge(rb[b], rb[b + 1]);
                else if (rc[b + 1]) rb[b] = rb[b + 1];
                rc[b] += rc[b + 1];
            }
            for (int b = 0; b < NB - 1; b++) {
                if (lc[b] == 0 || rc[b + 1] == 0) continue;
                float cost = lc[b] * area(lb[b]) / pA + rc[b + 1] * area(rb[b + 1]) / pA + 1.f;
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = ax;
                    float split_c = cmin + (b + 1.f) / NB * (cmax - cmin);
                    best_split = s;
                    for (int i = s; i < e; i++)
                        if (axis(cent[idx[i]], ax) < split_c) best_split++;
                    best_split = best_split <= s ? s + 1 : (best_split >= e ? e - 1 : best_split);
                }
            }
        }
        if (best_split <= s) best_split = s + 1;
        if (best_split >= e) best_split = e - 1;
        const int ba = best_axis;
        std::sort(idx.begin() + s, idx.begin() + e,
                  [&](int a, int b) { return axis(cent[a], ba) < axis(cent[b], ba); });
        int id = (int)nodes.size();
        nodes.push_back(nd);
        int l = rec(idx, s, best_split);
        int r = rec(idx, best_split, e);
        nodes[id].left = l;
        nodes[id].right = r;
        return id;
    }
};

// BVH4 node with fp16 bounds: layer/cuda_bvh_backend.cu:31-34
struct B4 { uint16_t bx[8], by[8], bz[8]; int child[4]; };
static_assert(sizeof(B4) == 64, "BVH4 node is 64 bytes");

uint16_t f2h(float f) {
    _Float16 h = (_Float16)f;  // IEEE binary16, round to nearest even
    uint16_t u;
    memcpy(&u, &h, 2);
    return u;
}

// collapseToB4: layer/cuda_bvh_backend.cu:391-418
int collapse_b4(const Builder& b2, int ni, B4* out, int& cnt) {
    const Node2& n = b2.nodes[ni];
    if (n.tri_count > 0) return -((n.tri_start << 3) | (n.tri_count - 1)) - 2;
    int gather[4], ng = 0;
    int ch[2] = {n.left, n.right};
    for (int c = 0; c < 2; c++) {
        const Node2& cn = b2.nodes[ch[c]];
        if (cn.tri_count > 0 || ng >= 3) { gather[ng++] = ch[c]; continue; }
        gather[ng++] = cn.left;
        gather[ng++] = cn.right;
    }
    B4 nd;
    for (int i = 0; i < 4; i++) {
        if (i < ng) {
            const Node2& cn = b2.nodes[gather[i]];
            nd.bx[i] = f2h(cn.box.mn.x); nd.bx[4 + i] = f2h(cn.box.mx.x);
            nd.by[i] = f2h(cn.box.mn.y); nd.by[4 + i] = f2h(cn.box.mx.y);
            nd.bz[i] = f2h(cn.box.mn.z); nd.bz[4 + i] = f2h(cn.box.mx.z);
        } else {
            nd.bx[i] = f2h(1e30f); nd.bx[4 + i] = f2h(-1e30f);
            nd.by[i] = f2h(1e30f); nd.by[4 + i] = f2h(-1e30f);
            nd.bz[i] = f2h(1e30f); nd.bz[4 + i] = f2h(-1e30f);
        }
        nd.child[i] = -1;
    }
    int me = cnt++;
    for (int i = 0; i < ng; i++) nd.child[i] = collapse_b4(b2, gather[i], out, cnt);
    out[me] = nd;
    return me;
}

// Preorder numbering + skip pointers: layer/cuda_bvh_backend.cu:462-522 (and
// the same two-pass scheme at :1632-1687 for the TLAS).  `boxes`, `is_leaf`,
// `left`, `right`, `leaf_enc` describe any binary tree rooted at node 0.
template <class NodeVec>
void dfs_export(const NodeVec& nodes, std::vector<uint32_t>& out) {
    struct Item { int idx, skip; };
    std::vector<int> order, skip;
    std::vector<Item> st;
    st.push_back({0, -1});
    while (!st.empty()) {
        Item it = st.back();
        st.pop_back();
        order.push_back(it.idx);
        skip.push_back(it.skip);
        const auto& n = nodes[it.idx];
        if (n.tri_count == 0) {
            st.push_back({n.right, it.skip});
            st.push_back({n.left, -2});
        }
    }
    int m = (int)order.size();
    std::vector<int> size(m, 1);
    for (int i = m - 1; i >= 0; i--) {
        const auto& n = nodes[order[i]];
        if (n.tri_count == 0) {
            int l = i + 1;
            size[i] = 1 + size[l];
            int r = i + 1 + size[l];
            if (r < m) size[i] += size[r];
            if (skip[l] == -2) skip[l] = r;
        }
    }
    out.assign((size_t)m * 8, 0u);
    for (int i = 0; i < m; i++) {
        const auto& n = nodes[order[i]];
        uint32_t* p = &out[(size_t)i * 8];
        memcpy(p + 0, &n.box.mn.x, 4); memcpy(p + 1, &n.box.mn.y, 4); memcpy(p + 2, &n.box.mn.z, 4);
        memcpy(p + 3, &n.box.mx.x, 4); memcpy(p + 4, &n.box.mx.y, 4); memcpy(p + 5, &n.box.mx.z, 4);
        int enc = n.tri_count > 0 ? -((n.tri_start << 3) | (n.tri_count - 1)) - 2 : 0;
        memcpy(p + 6, &enc, 4);
        memcpy(p + 7, &skip[i], 4);
    }
}

struct Handle {
    Builder b2;
    std::vector<uint32_t> dfs;
    std::vector<float> packed;
    std::vector<B4> b4;
    float center[3], extent;
};

// ---------------- Moller-Trumbore (layer/cuda_bvh_backend.cu:143-157) ----------------
// Returns true and (t,u,v) when the triangle passes all rejection tests; the
// caller applies the t-interval.  Every product and sum is one IEEE rounding.
inline bool mt(const float o[3], const float d[3], const float v0[3], const float e1[3],
               const float e2[3], float& t, float& u, float& v) {
    float px = d[1] * e2[2] - d[2] * e2[1];
    float py = d[2] * e2[0] - d[0] * e2[2];
    float pz = d[0] * e2[1] - d[1] * e2[0];
    float det = e1[0] * px + e1[1] * py + e1[2] * pz;
    if (fabsf(det) < 1e-12f) return false;
    float inv = 1.f / det;
    float sx = o[0] - v0[0], sy = o[1] - v0[1], sz = o[2] - v0[2];
    u = inv * (sx * px + sy * py + sz * pz);
    if (u < 0.f || u > 1.f) return false;
    float qx = sy * e1[2] - sz * e1[1];
    float qy = sz * e1[0] - sx * e1[2];
    float qz = sx * e1[1] - sy * e1[0];
    v = inv * (d[0] * qx + d[1] * qy + d[2] * qz);
    if (v < 0.f || u + v > 1.f) return false;
    t = inv * (e2[0] * qx + e2[1] * qy + e2[2] * qz);
    return true;
}

// Packed triangle i (layer/cuda_bvh_backend.cu:716-735): v0, v1, v2, orig id.
inline void unpack(const float* p, float v0[3], float e1[3], float e2[3], int& prim) {
    v0[0] = p[0]; v0[1] = p[1]; v0[2] = p[2];
    e1[0] = p[3] - p[0]; e1[1] = p[4] - p[1]; e1[2] = p[5] - p[2];
    e2[0] = p[6] - p[0]; e2[1] = p[7] - p[1]; e2[2] = p[8] - p[2];
    prim = (int)p[9];
}

// Conservative slab test, evaluated in double with a relative slack and a
// per-axis slack of 2^-20 of the box and origin coordinates times |1/d| (a
// grazing ray's accepted fp32 hit can lie that far outside the box), so the
// oracle never culls a box that holds an accepted fp32 hit.  Culling only
// affects speed; the hit set is defined by the triangle test alone.
struct DRay { double o[3], inv[3]; bool zero[3]; };
inline DRay dray(const float o[3], const float d[3]) {
    DRay r;
    for (int a = 0; a < 3; a++) {
        r.o[a] = o[a];
        r.zero[a] = (d[a] == 0.f);
        r.inv[a] = r.zero[a] ? 0.0 : 1.0 / (double)d[a];
    }
    return r;
}
inline bool box_hit(const DRay& r, const float* bmin, const float* bmax, double tmin, double tmax) {
    double tn = -INFINITY, tf = INFINITY;
    for (int a = 0; a < 3; a++) {
        double lo = bmin[a], hi = bmax[a];
        if (r.zero[a]) {
            double sl = 1e-7 * (fabs(lo) + fabs(hi)) + 1e-30;
            if (r.o[a] < lo - sl || r.o[a] > hi + sl) return false;
            continue;
        }
        double t1 = (lo - r.o[a]) * r.inv[a], t2 = (hi - r.o[a]) * r.inv[a];
        // per-axis slack for a ray nearly parallel to the slab: the fp32
        // triangle test's hit point may lie a few float roundings of the
        // coordinates outside the box, which 1/d turns into a large t
        const double ea = ldexp((fabs(lo) + fabs(hi) + 2.0 * fabs(r.o[a])) * fabs(r.inv[a]), -20);
        tn = std::max(tn, std::min(t1, t2) - ea);
        tf = std::min(tf, std::max(t1, t2) + ea);
    }
    double sl = 1e-5 * std::max(fabs(tn), fabs(tf)) + 1e-9;
    if (!(tn <= tf + sl)) return false;
    if (tf < tmin - sl) return false;
    if (tn > tmax + 1e-5 * fabs(tmax) + sl) return false;
    return true;
}

inline bool closer(float t, int prim, float best_t, int best_prim) {
    return t < best_t || (t == best_t && prim < best_prim);
}

// Stackless DFS traversal: layer/shaders/bvh2_stackless.comp:37-76.
// `any` stops at the first accepted triangle.  Returns the best hit.
template <bool ANY>
void trace_dfs_one(const uint32_t* dfs, int nnodes, const float* packed, const OrcRay& ray,
                   OrcHit& hit, uint64_t* st) {
    const float* o = ray.org;
    const float* d = ray.dir;
    DRay dr = dray(o, d);
    float best_t = ray.tmax;
    int best_p = -1;
    float bu = 0.f, bv = 0.f;
    uint64_t nvis = 0, ntri = 0;
    int ni = nnodes > 0 ? 0 : -1;
    while (ni >= 0 && ni < nnodes) {
        const uint32_t* w = dfs + (size_t)ni * 8;
        int leaf_enc, skip;
        memcpy(&leaf_enc, w + 6, 4);
        memcpy(&skip, w + 7, 4);
        float bmin[3], bmax[3];
        memcpy(bmin, w, 12);
        memcpy(bmax, w + 3, 12);
        bool hitbox = box_hit(dr, bmin, bmax, ray.tmin, best_t);
        if (!hitbox) { ni = skip; continue; }
        if (leaf_enc == 0) { nvis++; ni = ni + 1; continue; }
        int enc = -(leaf_enc + 2);
        int ts = enc >> 3, tc = (enc & 7) + 1;
        for (int k = 0; k < tc; k++) {
            float v0[3], e1[3], e2[3];
            int prim;
            unpack(packed + (size_t)(ts + k) * 12, v0, e1, e2, prim);
            float t, u, v;
            ntri++;
            if (!mt(o, d, v0, e1, e2, t, u, v)) continue;
            if (!(t > ray.tmin && t < ray.tmax)) continue;
            if (ANY) { best_p = prim; best_t = t; bu = u; bv = v; break; }
            if (best_p < 0 ? (t < best_t) : closer(t, prim, best_t, best_p)) {
                best_t = t; best_p = prim; bu = u; bv = v;
            }
        }
        if (ANY && best_p >= 0) break;
        ni = skip;
    }
    hit.t = best_p >= 0 ? best_t : INFINITY;
    hit.prim = best_p;
    hit.u = best_p >= 0 ? bu : 0.f;
    hit.v = best_p >= 0 ? bv : 0.f;
    if (st) { st[0] = nvis; st[1] = ntri; }
}

// Dynamic-chunk parallel loop over [0, n) on `nthreads` host threads
// (0 = all hardware threads).
template <class F>
void parallel_for(int n, int nthreads, int chunk, F fn) {
    int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
    if (nt < 1) nt = 1;
    if (nt == 1 || n <= chunk) {
        for (int i = 0; i < n; i++) fn(i);
        return;
    }
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            int s = next.fetch_add(chunk);
            if (s >= n) break;
            int e = std::min(n, s + chunk);
            for (int i = s; i < e; i++) fn(i);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
}

// ---------------- LBVH for TLAS (layer/cuda_bvh_backend.cu:257-389) ----------------
uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
uint32_t morton(float x, float y, float z) {
    x = fminf(fmaxf(x * 1024.0f, 0.0f), 1023.0f);
    y = fminf(fmaxf(y * 1024.0f, 0.0f), 1023.0f);
    z = fminf(fmaxf(z * 1024.0f, 0.0f), 1023.0f);
    return expand_bits((uint32_t)x) * 4 + expand_bits((uint32_t)y) * 2 + expand_bits((uint32_t)z);
}

struct LNode { Box box; int left, right, tri_start, tri_count; };

struct LBVH {
    std::vector<LNode> nodes;
    std::vector<int> ordered;
    std::vector<float> sorted;
    void build(const float* a, int n) {
        float smin[3] = {1e30f, 1e30f, 1e30f}, smax[3] = {-1e30f, -1e30f, -1e30f};
        for (int i = 0; i < n; i++)
            for (int k = 0; k < 3; k++) {
                float c = (a[i * 6 + k] + a[i * 6 + 3 + k]) * 0.5f;
                smin[k] = fminf(smin[k], c);
                smax[k] = fmaxf(smax[k], c);
            }
        float inv[3];
        for (int k = 0; k < 3; k++) inv[k] = (smax[k] - smin[k] > 1e-8f) ? 1.0f / (smax[k] - smin[k]) : 0.0f;
        std::vector<std::pair<uint32_t, int>> mp(n), tmp(n);
        for (int i = 0; i < n; i++) {
            float c[3];
            for (int k = 0; k < 3; k++) c[k] = (a[i * 6 + k] + a[i * 6 + 3 + k]) * 0.5f;
            mp[i] = {morton((c[0] - smin[0]) * inv[0], (c[1] - smin[1]) * inv[1], (c[2] - smin[2]) * inv[2]), i};
        }
        // stable LSD radix sort, 4 x 8 bits (same order as :309-324)
        for (int pass = 0; pass < 4; pass++) {
            int sh = pass * 8;
            int count[256] = {0}, pre[256];
            for (int i = 0; i < n; i++) count[(mp[i].first >> sh) & 0xFF]++;
            pre[0] = 0;
            for (int i = 1; i < 256; i++) pre[i] = pre[i - 1] + count[i - 1];
            for (int i = 0; i < n; i++) tmp[pre[(mp[i].first >> sh) & 0xFF]++] = mp[i];
            mp.swap(tmp);
        }
        ordered.resize(n);
        for (int i = 0; i < n; i++) ordered[i] = mp[i].second;
        sorted.resize((size_t)n * 6);
        for (int i = 0; i < n; i++)
            for (int k = 0; k < 6; k++) sorted[(size_t)i * 6 + k] = a[(size_t)ordered[i] * 6 + k];
        nodes.reserve((size_t)n * 2);
        rec(0, n);
    }
    int rec(int s, int e) {
        LNode nd;
        nd.left = nd.right = nd.tri_start = nd.tri_count = 0;
        nd.box.mn = {1e30f, 1e30f, 1e30f};
        nd.box.mx = {-1e30f, -1e30f, -1e30f};
        int cnt = e - s;
        if (cnt <= 1) {
            nd.tri_start = s;
            nd.tri_count = cnt;
            for (int i = s; i < e; i++) {
                nd.box.mn.x = fminf(nd.box.mn.x, sorted[i * 6 + 0]);
                nd.box.mn.y = fminf(nd.box.mn.y, sorted[i * 6 + 1]);
                nd.box.mn.z = fminf(nd.box.mn.z, sorted[i * 6 + 2]);
                nd.box.mx.x = fmaxf(nd.box.mx.x, sorted[i * 6 + 3]);
                nd.box.mx.y = fmaxf(nd.box.mx.y, sorted[i * 6 + 4]);
                nd.box.mx.z = fmaxf(nd.box.mx.z, sorted[i * 6 + 5]);
            }
            nodes.push_back(nd);
            return (int)nodes.size() - 1;
        }
        int mid = s + cnt / 2;
        int id = (int)nodes.size();
        nodes.push_back(nd);
        int l = rec(s, mid), r = rec(mid, e);
        nodes[id].left = l;
        nodes[id].right = r;
        const Box& L = nodes[l].box;
        const Box& R = nodes[r].box;
        nodes[id].box = merge(L, R);
        return id;
    }
};

// Instance ray transform: layer/rt_ir_exec.cu:81-91 (inverse 3x4, row major;
// the direction is not normalised, so t stays in world units).
inline void xform_ray(const float* inv, const float o[3], const float d[3], float lo[3], float ld[3]) {
    lo[0] = inv[0] * o[0] + inv[1] * o[1] + inv[2] * o[2] + inv[3];
    lo[1] = inv[4] * o[0] + inv[5] * o[1] + inv[6] * o[2] + inv[7];
    lo[2] = inv[8] * o[0] + inv[9] * o[1] + inv[10] * o[2] + inv[11];
    ld[0] = inv[0] * d[0] + inv[1] * d[1] + inv[2] * d[2];
    ld[1] = inv[4] * d[0] + inv[5] * d[1] + inv[6] * d[2];
    ld[2] = inv[8] * d[0] + inv[9] * d[1] + inv[10] * d[2];
}

// Two-level traversal (layer/rt_ir_exec.cu:93-189): TLAS leaves hold one
// instance each (layer/cuda_bvh_backend.cu:353-356); each instance's BLAS is
// walked in object space.  Ties break on (t, instance, prim).
template <bool ANY>
void trace_two_level_one(const uint32_t* tlas, int tn, const int* tord, const float* inv12,
                         const int* iblas, const uint32_t* bdfs, const int* noff, const float* bpk,
                         const int* toff, const OrcRay& ray, OrcHit& hit, int& inst_out) {
    DRay dr = dray(ray.org, ray.dir);
    float best_t = ray.tmax;
    int best_p = -1, best_i = -1;
    float bu = 0.f, bv = 0.f;
    int ni = tn > 0 ? 0 : -1;
    bool done = false;
    while (!done && ni >= 0 && ni < tn) {
        const uint32_t* w = tlas + (size_t)ni * 8;
        int leaf_enc, skip;
        memcpy(&leaf_enc, w + 6, 4);
        memcpy(&skip, w + 7, 4);
        float bmin[3], bmax[3];
        memcpy(bmin, w, 12);
        memcpy(bmax, w + 3, 12);
        if (!box_hit(dr, bmin, bmax, ray.tmin, best_t)) { ni = skip; continue; }
        if (leaf_enc == 0) { ni++; continue; }
        int enc = -(leaf_enc + 2);
        int ts = enc >> 3, tc = (enc & 7) + 1;
        for (int k = 0; k < tc && !done; k++) {
            int inst = tord[ts + k];
            int b = iblas[inst];
            float lo[3], ld[3];
            xform_ray(inv12 + (size_t)inst * 12, ray.org, ray.dir, lo, ld);
            DRay lr = dray(lo, ld);
            const uint32_t* nodes = bdfs + (size_t)noff[b] * 8;
            int nn = noff[b + 1] - noff[b];
            const float* pk = bpk + (size_t)toff[b] * 12;
            int bi = nn > 0 ? 0 : -1;
            while (bi >= 0 && bi < nn) {
                const uint32_t* bw = nodes + (size_t)bi * 8;
                int ble, bsk;
                memcpy(&ble, bw + 6, 4);
                memcpy(&bsk, bw + 7, 4);
                float mn[3], mx[3];
                memcpy(mn, bw, 12);
                memcpy(mx, bw + 3, 12);
                if (!box_hit(lr, mn, mx, ray.tmin, best_t)) { bi = bsk; continue; }
                if (ble == 0) { bi++; continue; }
                int be = -(ble + 2);
                int bts = be >> 3, btc = (be & 7) + 1;
                for (int j = 0; j < btc; j++) {
                    float v0[3], e1[3], e2[3];
                    int prim;
                    unpack(pk + (size_t)(bts + j) * 12, v0, e1, e2, prim);
                    float t, u, v;
                    if (!mt(lo, ld, v0, e1, e2, t, u, v)) continue;
                    if (!(t > ray.tmin && t < ray.tmax)) continue;
                    if (ANY) { best_p = prim; best_i = inst; best_t = t; done = true; break; }
                    bool better = best_p < 0 ? (t < best_t)
                                             : (t < best_t || (t == best_t && (inst < best_i ||
                                                (inst == best_i && prim < best_p))));
                    if (better) { best_t = t; best_p = prim; best_i = inst; bu = u; bv = v; }
                }
                if (done) break;
                bi = bsk;
            }
        }
        ni = skip;
    }
    hit.t = best_p >= 0 ? best_t : INFINITY;
    hit.prim = best_p;
    hit.u = best_p >= 0 ? bu : 0.f;
    hit.v = best_p >= 0 ? bv : 0.f;
    inst_out = best_i;
}

// ---------------- 8-wide compressed walk, with work counts ----------------
// The engine's own closest-hit / any-hit walk over its 8-wide nodes (the
// traceCWBVH scheme of cuda_rt_v37.cu:146-373: a node group is a child base
// plus an 8-bit hit mask, children taken in ray-octant order, child boxes
// quantised to 8 bits on the grid p + q * 2^e), restated step for step so
// that the node visits and triangle tests per ray -- the algorithmic bytes
// bench.py charges a launch -- and the results also come from the CPU.
//
// Node, 20 words:  [0..2] p (float), [3] exponent bytes x | y << 8 | z << 16
//   and the inner-child mask << 24, [4] first child node, [5] first triangle
//   record, [6] [7] one meta byte per slot 0-3 / 4-7 (inner 0xFF, leaf
//   count << 5 | offset, empty 0), [8..11] x planes (lo of slots 0-3, lo
//   4-7, hi 0-3, hi 4-7), [12..15] y, [16..19] z.
// Triangle record, 12 floats: v0 and the primitive id (int bits), e1, 0,
//   e2, 0.
// One round of the walk: up to `niters` node visits, then every triangle of
// the hit leaves is tested and the least (t, primitive) key kept, then the
// next group is popped if the current one is spent.  With `sets` = 1 a
// visit that gave triangles ends the round's visits, and a visited node
// with nothing hit pops the next group; with `sets` = 2 (the kernel's two
// pending triangle sets) the visits go on until a second visit has given
// triangles, and a spent group pops the next one after every visit.  Box test: t = q * (s / d) + (p - o) / d with an absolute
// slack of 2^-22 |(p - o) / d| on the offsets and 2^-21 |t_far| on the
// comparison; 1/d of a component with |d| <= 2^-64 uses +-2^-64.
struct Walk8Out {
    float t, u, v;
    int prim;
    uint8_t occ;
    uint32_t nodes, tris;
    bool bad;  // an index past the arrays (not a valid tree)
};

inline float as_f(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}
inline uint32_t ord_of(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
inline float from_ord(uint32_t u) { return as_f((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u); }
inline uint32_t bit_run(uint32_t start, uint32_t width) {
    return width ? (uint32_t)((((1ull << width) - 1ull) << start) & 0xFFFFFFFFull) : 0u;
}

void visit8(const uint32_t* W, const float o[3], const float inv[3], uint32_t oct, float tmin, float thit,
            uint32_t& tri_base, uint32_t& tmask, uint32_t& ngx, uint32_t& ngy) {
    const uint32_t e = W[3], imask = e >> 24;
    float S[3], On[3], Of[3];
    for (int a = 0; a < 3; a++) {
        const float sc = as_f(((e >> (8 * a)) & 0xFFu) << 23);
        S[a] = sc * inv[a];
        const float O = (as_f(W[a]) - o[a]) * inv[a];
        On[a] = fmaf(-fabsf(O), 0x1p-22f, O);
        Of[a] = fmaf(fabsf(O), 0x1p-22f, O);
    }
    uint32_t nh = 0, th = 0;
    for (int s = 0; s < 8; s++) {
        float tn[3], tf[3];
        for (int a = 0; a < 3; a++) {
            const uint32_t* P = W + 8 + 4 * a;
            const bool neg = (oct >> a) & 1u;  // near plane: lo for a positive 1/d, hi otherwise
            const uint32_t nw = neg ? P[2 + (s >> 2)] : P[s >> 2];
            const uint32_t fw = neg ? P[s >> 2] : P[2 + (s >> 2)];
            tn[a] = fmaf((float)((nw >> (8 * (s & 3))) & 0xFFu), S[a], On[a]);
            tf[a] = fmaf((float)((fw >> (8 * (s & 3))) & 0xFFu), S[a], Of[a]);
        }
        const float tnear = fmaxf(fmaxf(tn[0], tn[1]), fmaxf(tn[2], tmin));
        const float tfar = fminf(fminf(tf[0], tf[1]), fminf(tf[2], thit));
        if (!(tnear <= fmaf(fabsf(tfar), 0x1p-21f, tfar))) continue;
        if ((imask >> s) & 1u) {
            nh |= 1u << ((uint32_t)s ^ oct);
        } else {
            const uint32_t meta = (W[6 + (s >> 2)] >> (8 * (s & 3))) & 0xFFu;
            th |= bit_run(meta & 31u, meta >> 5);
        }
    }
    tri_base = W[5];
    tmask = th;
    ngx = W[4];
    ngy = nh | (imask << 8);
}

void walk8_one(const uint32_t* nodes, int nnodes, const float* recs, int nrecs, const OrcRay& ray, bool any,
               int niters, int sets, Walk8Out& out) {
    const float* o = ray.org;
    const float* d = ray.dir;
    float inv[3];
    for (int a = 0; a < 3; a++) inv[a] = 1.0f / (fabsf(d[a]) > 0x1p-64f ? d[a] : copysignf(0x1p-64f, d[a]));
    const uint32_t oct =
        (std::signbit(inv[0]) ? 1u : 0u) | (std::signbit(inv[1]) ? 2u : 0u) | (std::signbit(inv[2]) ? 4u : 0u);
    float thit = ray.tmax, hu = 0.f, hv = 0.f;
    int hprim = -1;
    uint32_t cn = 0, ct = 0;
    uint32_t stx[64], sty[64];
    int sp = 0;
    bool overflow = false, found = false;
    uint32_t ngx = 0, ngy = (1u << oct) | (1u << 8);  // the root as slot 0 of a one-child group
    out.bad = false;
    for (;;) {
        uint32_t tri_base = 0, tmask = 0, tri_base2 = 0, tmask2 = 0;
        for (int it = 0; it < niters; it++) {
            if ((sets == 2 ? tmask2 : tmask) != 0 || overflow || (ngy & 0xFFu) == 0) continue;
            uint32_t hitsm = ngy & 0xFFu;
            const uint32_t imask = (ngy >> 8) & 0xFFu;
            const uint32_t k = (uint32_t)__builtin_ctz(hitsm);
            hitsm &= hitsm - 1;
            const uint32_t slot = k ^ oct;
            const uint32_t ni = ngx + (uint32_t)__builtin_popcount(imask & ((1u << slot) - 1u));
            if (hitsm) {
                if (sp < 64) {
                    stx[sp] = ngx;
                    sty[sp] = hitsm | (imask << 8);
                    sp++;
                } else {
                    overflow = true;
                }
            }
            cn++;
            if (ni >= (uint32_t)nnodes) {
                out.bad = true;
                return;
            }
            uint32_t vb, vm;
            visit8(nodes + (size_t)ni * 20, o, inv, oct, ray.tmin, thit, vb, vm, ngx, ngy);
            if (tmask == 0) {
                tri_base = vb;
                tmask = vm;
            } else {
                tri_base2 = vb;
                tmask2 = vm;
            }
            if (niters > 1 && (sets == 2 || tmask == 0) && (ngy & 0xFFu) == 0 && sp > 0) {
                sp--;
                ngx = stx[sp];
                ngy = sty[sp];
            }
        }
        ct += (uint32_t)__builtin_popcount(tmask) + (uint32_t)__builtin_popcount(tmask2);
        if (tmask | tmask2) {
            uint64_t best = ((uint64_t)ord_of(thit) << 32) | (uint32_t)(hprim >= 0 ? hprim : -1);
            float bu = 0.f, bv = 0.f;
            bool improved = false;
            for (uint64_t m = (uint64_t)tmask | ((uint64_t)tmask2 << 32); m; m &= m - 1) {
                const int bit = __builtin_ctzll(m);
                const uint32_t rec = (bit < 32 ? tri_base : tri_base2) + (uint32_t)(bit & 31);
                if (rec >= (uint32_t)nrecs) {
                    out.bad = true;
                    return;
                }
                const float* R = recs + (size_t)rec * 12;
                float t, u, v;
                if (!mt(o, d, R, R + 4, R + 8, t, u, v) || !(t > ray.tmin && t < ray.tmax)) continue;
                if (any) {
                    found = true;
                } else {
                    uint32_t pid;
                    memcpy(&pid, R + 3, 4);
                    const uint64_t key = ((uint64_t)ord_of(t) << 32) | pid;
                    if (key < best) {
                        best = key;
                        bu = u;
                        bv = v;
                        improved = true;
                    }
                }
            }
            if (improved) {
                thit = from_ord((uint32_t)(best >> 32));
                hprim = (int)(uint32_t)best;
                hu = bu;
                hv = bv;
            }
        }
        bool done = overflow || (any && found);
        if (!done && (ngy & 0xFFu) == 0) {
            if (sp == 0) {
                done = true;
            } else {
                sp--;
                ngx = stx[sp];
                ngy = sty[sp];
            }
        }
        if (done) {
            if (overflow) {
                hprim = -1;
                found = false;
            }
            out.t = hprim >= 0 ? thit : INFINITY;
            out.prim = hprim;
            out.u = hprim >= 0 ? hu : 0.f;
            out.v = hprim >= 0 ? hv : 0.f;
            out.occ = found ? 1 : 0;
            out.nodes = cn;
            out.tris = ct;
            return;
        }
    }
}

}  // namespace

extern "C" {

void* orc_build(const float* tris9, int n, int nbins, int max_leaf) {
    if (!tris9 || n <= 0) return nullptr;
    Handle* h = new Handle();
    const Tri* t = reinterpret_cast<const Tri*>(tris9);
    h->b2.nbins = nbins;
    h->b2.max_leaf = max_leaf;
    h->b2.build(t, n);
    dfs_export(h->b2.nodes, h->dfs);
    int no = (int)h->b2.ordered.size();
    h->packed.assign((size_t)no * 12, 0.f);
    for (int i = 0; i < no; i++) {
        float* p = &h->packed[(size_t)i * 12];
        const Tri& tr = h->b2.ordered[i];
        p[0] = tr.v0.x; p[1] = tr.v0.y; p[2] = tr.v0.z; p[3] = tr.v1.x;
        p[4] = tr.v1.y; p[5] = tr.v1.z; p[6] = tr.v2.x; p[7] = tr.v2.y;
        p[8] = tr.v2.z; p[9] = (float)h->b2.orig[i]; p[10] = 0.f; p[11] = 0.f;
    }
    h->b4.resize(h->b2.nodes.size());
    int cnt = 0;
    collapse_b4(h->b2, 0, h->b4.data(), cnt);
    h->b4.resize(cnt);
    float bmin[3] = {1e30f, 1e30f, 1e30f}, bmax[3] = {-1e30f, -1e30f, -1e30f};
    for (int i = 0; i < n; i++)
        for (int a = 0; a < 3; a++) {
            const float* tt = tris9 + (size_t)i * 9;
            bmin[a] = std::min({bmin[a], tt[a], tt[3 + a], tt[6 + a]});
            bmax[a] = std::max({bmax[a], tt[a], tt[3 + a], tt[6 + a]});
        }
    for (int a = 0; a < 3; a++) h->center[a] = (bmin[a] + bmax[a]) * 0.5f;
    float ex = bmax[0] - bmin[0], ey = bmax[1] - bmin[1], ez = bmax[2] - bmin[2];
    h->extent = sqrtf(ex * ex + ey * ey + ez * ez);
    return h;
}
void orc_free(void* h) { delete static_cast<Handle*>(h); }
int orc_num_bvh2(void* h) { return (int)static_cast<Handle*>(h)->b2.nodes.size(); }
int orc_num_dfs(void* h) { return (int)(static_cast<Handle*>(h)->dfs.size() / 8); }
const uint32_t* orc_dfs(void* h) { return static_cast<Handle*>(h)->dfs.data(); }
int orc_num_packed(void* h) { return (int)(static_cast<Handle*>(h)->packed.size() / 4); }
const float* orc_packed(void* h) { return static_cast<Handle*>(h)->packed.data(); }
int orc_num_bvh4(void* h) { return (int)static_cast<Handle*>(h)->b4.size(); }
const void* orc_bvh4(void* h) { return static_cast<Handle*>(h)->b4.data(); }
const int* orc_orig_idx(void* h) { return static_cast<Handle*>(h)->b2.orig.data(); }
void orc_bounds(void* hv, float* cx, float* cy, float* cz, float* extent) {
    Handle* h = static_cast<Handle*>(hv);
    *cx = h->center[0]; *cy = h->center[1]; *cz = h->center[2]; *extent = h->extent;
}

int orc_tlas_fast(const float* aabbs, int n, uint32_t** out_nodes, int** out_ordered) {
    if (!aabbs || n <= 0 || !out_nodes) return 0;
    LBVH l;
    l.build(aabbs, n);
    std::vector<uint32_t> d;
    dfs_export(l.nodes, d);
    *out_nodes = (uint32_t*)malloc(d.size() * 4);
    memcpy(*out_nodes, d.data(), d.size() * 4);
    if (out_ordered) {
        *out_ordered = (int*)malloc((size_t)n * 4);
        memcpy(*out_ordered, l.ordered.data(), (size_t)n * 4);
    }
    return (int)(d.size() / 8);
}
void orc_free_ptr(void* p) { free(p); }

void orc_trace_closest_dfs(const uint32_t* dfs, int nnodes, const float* packed, const OrcRay* rays,
                           int nrays, OrcHit* hits, int nthreads, uint64_t* stats) {
    parallel_for(nrays, nthreads, 256, [&](int i) {
        trace_dfs_one<false>(dfs, nnodes, packed, rays[i], hits[i], stats ? stats + (size_t)i * 2 : nullptr);
    });
}

void orc_trace_any_dfs(const uint32_t* dfs, int nnodes, const float* packed, const OrcRay* rays,
                       int nrays, uint8_t* occ, int nthreads) {
    parallel_for(nrays, nthreads, 256, [&](int i) {
        OrcHit h;
        trace_dfs_one<true>(dfs, nnodes, packed, rays[i], h, nullptr);
        occ[i] = h.prim >= 0 ? 1 : 0;
    });
}

void orc_brute_closest(const float* tris9, int ntris, const OrcRay* rays, int nrays, OrcHit* hits,
                       int nthreads) {
    parallel_for(nrays, nthreads, 16, [&](int i) {
        const OrcRay& r = rays[i];
        float bt = r.tmax, bu = 0.f, bv = 0.f;
        int bp = -1;
        for (int k = 0; k < ntris; k++) {
            const float* p = tris9 + (size_t)k * 9;
            float v0[3] = {p[0], p[1], p[2]};
            float e1[3] = {p[3] - p[0], p[4] - p[1], p[5] - p[2]};
            float e2[3] = {p[6] - p[0], p[7] - p[1], p[8] - p[2]};
            float t, u, v;
            if (!mt(r.org, r.dir, v0, e1, e2, t, u, v)) continue;
            if (!(t > r.tmin && t < r.tmax)) continue;
            if (bp < 0 ? t < bt : closer(t, k, bt, bp)) { bt = t; bp = k; bu = u; bv = v; }
        }
        hits[i].t = bp >= 0 ? bt : INFINITY;
        hits[i].prim = bp;
        hits[i].u = bp >= 0 ? bu : 0.f;
        hits[i].v = bp >= 0 ? bv : 0.f;
    });
}

void orc_brute_any(const float* tris9, int ntris, const OrcRay* rays, int nrays, uint8_t* occ,
                   int nthreads) {
    parallel_for(nrays, nthreads, 16, [&](int i) {
        const OrcRay& r = rays[i];
        uint8_t o = 0;
        for (int k = 0; k < ntris && !o; k++) {
            const float* p = tris9 + (size_t)k * 9;
            float v0[3] = {p[0], p[1], p[2]};
            float e1[3] = {p[3] - p[0], p[4] - p[1], p[5] - p[2]};
            float e2[3] = {p[6] - p[0], p[7] - p[1], p[8] - p[2]};
            float t, u, v;
            if (mt(r.org, r.dir, v0, e1, e2, t, u, v) && t > r.tmin && t < r.tmax) o = 1;
        }
        occ[i] = o;
    });
}

void orc_trace_closest_two_level(const uint32_t* tlas, int tlas_nodes, const int* tlas_ordered,
                                 const float* inv12, const int* inst_blas, int ninst,
                                 const uint32_t* blas_dfs, const int* node_off,
                                 const float* blas_packed, const int* tri_off, const OrcRay* rays,
                                 int nrays, OrcHit* hits, int32_t* inst_out, int nthreads) {
    (void)ninst;
    parallel_for(nrays, nthreads, 64, [&](int i) {
        int inst;
        trace_two_level_one<false>(tlas, tlas_nodes, tlas_ordered, inv12, inst_blas, blas_dfs, node_off,
                                   blas_packed, tri_off, rays[i], hits[i], inst);
        if (inst_out) inst_out[i] = inst;
    });
}

void orc_trace_any_two_level(const uint32_t* tlas, int tlas_nodes, const int* tlas_ordered,
                             const float* inv12, const int* inst_blas, int ninst,
                             const uint32_t* blas_dfs, const int* node_off, const float* blas_packed,
                             const int* tri_off, const OrcRay* rays, int nrays, uint8_t* occ,
                             int nthreads) {
    (void)ninst;
    parallel_for(nrays, nthreads, 64, [&](int i) {
        OrcHit h;
        int inst;
        trace_two_level_one<true>(tlas, tlas_nodes, tlas_ordered, inv12, inst_blas, blas_dfs, node_off,
                                  blas_packed, tri_off, rays[i], h, inst);
        occ[i] = h.prim >= 0 ? 1 : 0;
    });
}

// Philox4x32-10, Salmon et al., "Parallel random numbers: as easy as 1, 2, 3" (SC'11).
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

uint16_t orc_f2h_rn(float f) { return f2h(f); }

// Recompute every skip pointer of a stackless DFS export from the tree shape
// (inner node i: left child i+1, right child i+1+size(left)); skip(i) is the
// first index after i's subtree, -1 past the end.  The reference's two-pass
// export (layer/cuda_bvh_backend.cu:488-503, :1652-1663) only resolves the
// placeholder of left children, so the right descendants of a left child keep
// skip == -2 and a stackless walk stops there.  The byte-identical
// restatement above keeps that behaviour; traversal parity uses this fix.
int orc_fix_skips(uint32_t* dfs, int n) {
    std::vector<int> size(n, 1);
    for (int i = n - 1; i >= 0; i--) {
        int le;
        memcpy(&le, dfs + (size_t)i * 8 + 6, 4);
        if (le == 0) {
            int l = i + 1;
            if (l >= n) return -1;
            int r = l + size[l];
            if (r >= n) return -1;
            size[i] = 1 + size[l] + size[r];
        }
    }
    int changed = 0;
    for (int i = 0; i < n; i++) {
        int sk = i + size[i] < n ? i + size[i] : -1;
        int old;
        memcpy(&old, dfs + (size_t)i * 8 + 7, 4);
        if (old != sk) changed++;
        memcpy(dfs + (size_t)i * 8 + 7, &sk, 4);
    }
    return changed;
}

// 8-wide walk over the engine's own nodes (walk8_one): `niters` node visits
// per round and `sets` (1 or 2) pending triangle sets per ray.  hits
// (closest hit) or occluded (any hit) may be null; counts: node visits and
// triangle tests per ray (2 x u32).  Returns how many rays' walks left the
// arrays (0 for a valid tree; those rays get counts 0xFFFFFFFF), or -1 for
// a bad niters / sets.
int orc_walk_bvh8(const uint32_t* nodes, int nnodes, const float* recs, int nrecs, const OrcRay* rays, int nrays,
                  int any, int niters, int sets, OrcHit* hits, uint8_t* occluded, uint32_t* counts, int nthreads) {
    if (sets < 1 || sets > 2 || niters < 1) return -1;
    std::atomic<int> bad(0);
    parallel_for(nrays, nthreads, 256, [&](int i) {
        Walk8Out w;
        walk8_one(nodes, nnodes, recs, nrecs, rays[i], any != 0, niters, sets, w);
        if (w.bad) {
            bad.fetch_add(1);
            w = Walk8Out{INFINITY, 0.f, 0.f, -1, 0, 0xFFFFFFFFu, 0xFFFFFFFFu, true};
        }
        if (hits) hits[i] = OrcHit{w.t, w.prim, w.u, w.v};
        if (occluded) occluded[i] = w.occ;
        if (counts) {
            counts[2 * i] = w.nodes;
            counts[2 * i + 1] = w.tris;
        }
    });
    return bad.load();
}

// ---- next-bounce ray generation, restating the library's
// cudaBVH_generateRays (itself after genAndCompact, multi_bounce.cu:281-362:
// hit point, facing geometric normal, tangent frame branching on the larger
// of |nx| |ny|, origin offset eps * n).  Every step is one correctly rounded
// single-precision operation in the same order as the GPU (this file is
// compiled with -ffp-contract=off); random numbers are Philox4x32-10 with
// key (seed, 3) for diffuse and (seed, 4) for shadow rays and counter
// (output index, block, 0, 0); the cosine-weighted direction is Malley's
// method on the first of eight uniform points of [-1,1)^2 inside the unit
// disk.  Survivors (hits whose primitive is < ntris) keep input order.
static inline float gen_u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

static void gen_one_ray(const float* tris9, const OrcRay& ray, const OrcHit& h, uint32_t item, int kind,
                        uint32_t seed, float eps, float tmin, float tmax, const float* lc, float lsize,
                        OrcRay& r) {
    const float px = ray.org[0] + h.t * ray.dir[0], py = ray.org[1] + h.t * ray.dir[1],
                pz = ray.org[2] + h.t * ray.dir[2];
    const float* v = tris9 + (size_t)h.prim * 9;
    const float e1x = v[3] - v[0], e1y = v[4] - v[1], e1z = v[5] - v[2];
    const float e2x = v[6] - v[0], e2y = v[7] - v[1], e2z = v[8] - v[2];
    float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    const float nl = 1.0f / sqrtf(fmaxf(nx * nx + ny * ny + nz * nz, 1e-30f));
    nx = nx * nl;
    ny = ny * nl;
    nz = nz * nl;
    if (nx * ray.dir[0] + ny * ray.dir[1] + nz * ray.dir[2] > 0.f) {
        nx = -nx;
        ny = -ny;
        nz = -nz;
    }
    const float ox = px + eps * nx, oy = py + eps * ny, oz = pz + eps * nz;
    r.org[0] = ox;
    r.org[1] = oy;
    r.org[2] = oz;
    const uint32_t key[2] = {seed, kind == 0 ? 3u : 4u};
    if (kind == 0) {
        float tx, ty, tz;
        if (fabsf(nx) > fabsf(ny)) {
            const float il = 1.0f / sqrtf(nx * nx + nz * nz);
            tx = -nz * il;
            ty = 0.f;
            tz = nx * il;
        } else {
            const float il = 1.0f / sqrtf(ny * ny + nz * nz);
            tx = 0.f;
            ty = nz * il;
            tz = -ny * il;
        }
        const float bx = ny * tz - nz * ty, by = nz * tx - nx * tz, bz = nx * ty - ny * tx;
        float x = 0.f, y = 0.f;
        for (uint32_t blk = 0; blk < 4; blk++) {
            const uint32_t ctr[4] = {item, blk, 0u, 0u};
            uint32_t b[4];
            orc_philox4x32_10(ctr, key, b);
            const float a0 = 2.f * gen_u01(b[0]) - 1.f, b0 = 2.f * gen_u01(b[1]) - 1.f;
            const float a1 = 2.f * gen_u01(b[2]) - 1.f, b1 = 2.f * gen_u01(b[3]) - 1.f;
            if (a0 * a0 + b0 * b0 < 1.f) {
                x = a0;
                y = b0;
                break;
            }
            if (a1 * a1 + b1 * b1 < 1.f) {
                x = a1;
                y = b1;
                break;
            }
        }
        const float z = sqrtf(fmaxf(1.f - x * x - y * y, 0.f));
        const float dx = x * tx + y * bx + z * nx, dy = x * ty + y * by + z * ny, dz = x * tz + y * bz + z * nz;
        const float dl = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
        r.dir[0] = dx * dl;
        r.dir[1] = dy * dl;
        r.dir[2] = dz * dl;
        r.tmin = tmin;
        r.tmax = tmax;
    } else {
        const uint32_t ctr[4] = {item, 0u, 0u, 0u};
        uint32_t b[4];
        orc_philox4x32_10(ctr, key, b);
        const float lx = lc[0] + (gen_u01(b[0]) - 0.5f) * lsize, ly = lc[1], lz = lc[2] + (gen_u01(b[1]) - 0.5f) * lsize;
        const float dx = lx - ox, dy = ly - oy, dz = lz - oz;
        const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
        r.dir[0] = dx / dist;
        r.dir[1] = dy / dist;
        r.dir[2] = dz / dist;
        r.tmin = tmin;
        r.tmax = dist * 0.9999f;
    }
}

// Returns the number of rays written (count if count > 0 and there are hits,
// the number of hits if count == 0).
int orc_generate_rays(const float* tris9, int ntris, const OrcRay* rays, const OrcHit* hits, int n, int kind,
                      int count, uint32_t seed, float eps, float tmin, float tmax, const float* light_center,
                      float light_size, OrcRay* out, int32_t* src, int nthreads) {
    std::vector<int> surv;
    surv.reserve(n);
    for (int i = 0; i < n; i++)
        if (hits[i].prim >= 0 && hits[i].prim < ntris) surv.push_back(i);
    const int m = (int)surv.size();
    const int total = m == 0 ? 0 : (count > 0 ? count : m);
    parallel_for(total, nthreads, 4096, [&](int k) {
        const int s = surv[k % m];
        gen_one_ray(tris9, rays[s], hits[s], (uint32_t)k, kind, seed, eps, tmin, tmax, light_center, light_size,
                    out[k]);
        if (src) src[k] = s;
    });
    return total;
}


}  // extern "C"

// ===================== FP64 path-tracing oracle =====================
// Mirrors the wavefront path tracer's model step by step (camera, hit
// frame, next-event estimation with an exact integer light CDF, Malley
// bounce, Russian roulette).  Every geometric quantity and every decision
// uses the same fp32 operations as the GPU (this file is compiled with
// -ffp-contract=off), so the paths are the same; radiance is accumulated
// in double.
namespace {

const uint32_t kPtKey = 0x50545201u;

inline void pt_rand(uint32_t pixel, uint32_t s, uint32_t b, uint32_t purpose, uint32_t seed, uint32_t out[4]) {
    const uint32_t ctr[4] = {pixel, s, (b << 8) | purpose, 0u};
    const uint32_t key[2] = {seed, kPtKey};
    orc_philox4x32_10(ctr, key, out);
}
inline float u01f(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }
inline float dot3f(float ax, float ay, float az, float bx, float by, float bz) { return ax * bx + ay * by + az * bz; }
inline void xpoint(const float* m, float x, float y, float z, float& ox, float& oy, float& oz) {
    ox = m[0] * x + m[1] * y + m[2] * z + m[3];
    oy = m[4] * x + m[5] * y + m[6] * z + m[7];
    oz = m[8] * x + m[9] * y + m[10] * z + m[11];
}

double tri_area_world_d(const float* m, const float* v) {
    double p[3][3];
    for (int k = 0; k < 3; k++)
        for (int r = 0; r < 3; r++)
            p[k][r] = (double)m[r * 4] * v[k * 3] + (double)m[r * 4 + 1] * v[k * 3 + 1] +
                      (double)m[r * 4 + 2] * v[k * 3 + 2] + (double)m[r * 4 + 3];
    const double a[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    const double b[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    const double c[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    return 0.5 * sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
}

}  // namespace

extern "C" {



void orc_pt_pixels(const OrcPTScene* S, const float* cam, const OrcPTParams* P, const int* pixels, int npix,
                   double* out_rgb, int nthreads, uint64_t* ray_counts) {
    // light table: emissive instances in order, their primitives in order
    std::vector<double> areas;
    std::vector<std::pair<int, int>> lights;
    for (int k = 0; k < S->ninst; k++) {
        const float* e = S->emission3 + 3 * k;
        if (!(e[0] > 0.f || e[1] > 0.f || e[2] > 0.f)) continue;
        const int b = S->inst_blas[k];
        for (int p = 0; p < S->blas_tri_count[b]; p++) {
            areas.push_back(tri_area_world_d(S->fwd12 + 12 * k, S->blas_tris9 + (size_t)(S->blas_tri_base[b] + p) * 9));
            lights.push_back({k, p});
        }
    }
    std::vector<unsigned long long> cdf(areas.size());
    unsigned long long total_q = 0;
    double light_area = 0.0;
    if (!areas.empty()) {
        double amax = 0.0;
        for (double a : areas) amax = std::max(amax, a);
        const int K = (int)floor(61.0 - log2((double)areas.size() * std::max(amax, 1e-300)));
        for (size_t i = 0; i < areas.size(); i++) {
            total_q += (unsigned long long)floor(ldexp(areas[i], K));
            cdf[i] = total_q;
        }
        light_area = ldexp((double)total_q, -K);
    }
    const float* eye = cam; const float* F = cam + 3; const float* R = cam + 6; const float* U = cam + 9;
    const float th = cam[12], aspect = cam[13];
    const int W = P->width, H = P->height, spp = P->spp;
    std::atomic<uint64_t> n_ext(0), n_sha(0);
    parallel_for(npix, nthreads, 1, [&](int ip) {
        const uint32_t pixel = (uint32_t)pixels[ip];
        const uint32_t px = pixel % W, py = pixel / W;
        double acc[3] = {0, 0, 0};
        uint64_t ne = 0, ns = 0;
        for (int s = 0; s < spp; s++) {
            uint32_t rr[4];
            pt_rand(pixel, s, 0, 0, P->seed, rr);
            const float j1 = u01f(rr[0]), j2 = u01f(rr[1]);
            const float x = (((float)px + j1) / (float)W * 2.f - 1.f) * th * aspect;
            const float y = (1.f - ((float)py + j2) / (float)H * 2.f) * th;
            float dx = F[0] + x * R[0] + y * U[0];
            float dy = F[1] + x * R[1] + y * U[1];
            float dz = F[2] + x * R[2] + y * U[2];
            const float len = sqrtf(dot3f(dx, dy, dz, dx, dy, dz));
            OrcRay ray;
            ray.org[0] = eye[0]; ray.org[1] = eye[1]; ray.org[2] = eye[2]; ray.tmin = 0.f;
            ray.dir[0] = dx / len; ray.dir[1] = dy / len; ray.dir[2] = dz / len; ray.tmax = 1e30f;
            float tpf[3] = {1.f, 1.f, 1.f};
            double tpd[3] = {1.0, 1.0, 1.0};
            double L[3] = {0, 0, 0};
            for (int b = 0; b < P->max_bounces; b++) {
                OrcHit h;
                int inst = -1;
                ne++;
                trace_two_level_one<false>(S->tlas, S->tlas_nodes, S->tlas_ordered, S->inv12, S->inst_blas,
                                           S->blas_dfs, S->node_off, S->blas_packed, S->tri_off, ray, h, inst);
                if (h.prim < 0) break;
                const float* alb = S->albedo3 + 3 * inst;
                const float* emi = S->emission3 + 3 * inst;
                if (b == 0 && (emi[0] > 0.f || emi[1] > 0.f || emi[2] > 0.f))
                    for (int c = 0; c < 3; c++) L[c] += tpd[c] * (double)emi[c];
                const float hx = ray.org[0] + h.t * ray.dir[0];
                const float hy = ray.org[1] + h.t * ray.dir[1];
                const float hz = ray.org[2] + h.t * ray.dir[2];
                const int bl = S->inst_blas[inst];
                const float* tv = S->blas_tris9 + (size_t)(S->blas_tri_base[bl] + h.prim) * 9;
                const float e1x = tv[3] - tv[0], e1y = tv[4] - tv[1], e1z = tv[5] - tv[2];
                const float e2x = tv[6] - tv[0], e2y = tv[7] - tv[1], e2z = tv[8] - tv[2];
                const float nox = e1y * e2z - e1z * e2y, noy = e1z * e2x - e1x * e2z, noz = e1x * e2y - e1y * e2x;
                const float* iv = S->inv12 + 12 * inst;
                float nx = iv[0] * nox + iv[4] * noy + iv[8] * noz;
                float ny = iv[1] * nox + iv[5] * noy + iv[9] * noz;
                float nz = iv[2] * nox + iv[6] * noy + iv[10] * noz;
                const float nl = sqrtf(dot3f(nx, ny, nz, nx, ny, nz));
                nx = nx / nl; ny = ny / nl; nz = nz / nl;
                if (dot3f(nx, ny, nz, ray.dir[0], ray.dir[1], ray.dir[2]) > 0.f) { nx = -nx; ny = -ny; nz = -nz; }
                const float ox = hx + 1e-3f * nx, oy = hy + 1e-3f * ny, oz = hz + 1e-3f * nz;
                if (!lights.empty()) {
                    uint32_t rl[4];
                    pt_rand(pixel, s, b, 1, P->seed, rl);
                    const unsigned long long r64 = ((unsigned long long)rl[0] << 32) | rl[1];
                    const unsigned long long target = (unsigned long long)(((unsigned __int128)r64 * total_q) >> 64);
                    const size_t li = std::upper_bound(cdf.begin(), cdf.end(), target) - cdf.begin();
                    const int linst = lights[li].first, lprim = lights[li].second;
                    const int lb = S->inst_blas[linst];
                    const float* lv = S->blas_tris9 + (size_t)(S->blas_tri_base[lb] + lprim) * 9;
                    const float* fw = S->fwd12 + 12 * linst;
                    float ax, ay, az, bx, by, bz, cx, cy, cz;
                    xpoint(fw, lv[0], lv[1], lv[2], ax, ay, az);
                    xpoint(fw, lv[3], lv[4], lv[5], bx, by, bz);
                    xpoint(fw, lv[6], lv[7], lv[8], cx, cy, cz);
                    const float su = sqrtf(u01f(rl[2])), xb = u01f(rl[3]);
                    const float wa = 1.f - su, wb = su * (1.f - xb), wc = su * xb;
                    const float lx = wa * ax + wb * bx + wc * cx;
                    const float ly = wa * ay + wb * by + wc * cy;
                    const float lz = wa * az + wb * bz + wc * cz;
                    const float f1x = bx - ax, f1y = by - ay, f1z = bz - az;
                    const float f2x = cx - ax, f2y = cy - ay, f2z = cz - az;
                    const float gx = f1y * f2z - f1z * f2y, gy = f1z * f2x - f1x * f2z, gz = f1x * f2y - f1y * f2x;
                    const float gl = sqrtf(dot3f(gx, gy, gz, gx, gy, gz));
                    const float tx = lx - ox, ty = ly - oy, tz = lz - oz;
                    const float d2 = dot3f(tx, ty, tz, tx, ty, tz);
                    const float dist = sqrtf(d2);
                    if (dist > 0.f && gl > 0.f) {
                        const float sdx = tx / dist, sdy = ty / dist, sdz = tz / dist;
                        const float cxf = dot3f(nx, ny, nz, sdx, sdy, sdz);
                        const float clf = fabsf(dot3f(gx, gy, gz, sdx, sdy, sdz)) / gl;
                        if (cxf > 0.f && clf > 0.f) {
                            OrcRay sr;
                            sr.org[0] = ox; sr.org[1] = oy; sr.org[2] = oz; sr.tmin = 1e-4f;
                            sr.dir[0] = sdx; sr.dir[1] = sdy; sr.dir[2] = sdz; sr.tmax = dist * 0.9999f;
                            OrcHit sh;
                            int sinst;
                            ns++;
                            trace_two_level_one<true>(S->tlas, S->tlas_nodes, S->tlas_ordered, S->inv12, S->inst_blas,
                                                      S->blas_dfs, S->node_off, S->blas_packed, S->tri_off, sr, sh,
                                                      sinst);
                            if (sh.prim < 0) {
                                const float* le = S->emission3 + 3 * linst;
                                const double g = (double)cxf * (double)clf / (double)d2 * light_area / M_PI;
                                for (int c = 0; c < 3; c++) L[c] += tpd[c] * (double)alb[c] * (double)le[c] * g;
                            }
                        }
                    }
                }
                if (b + 1 >= P->max_bounces) break;
                float tfx, tfy, tfz;
                if (fabsf(nx) > fabsf(ny)) {
                    const float il = 1.f / sqrtf(nx * nx + nz * nz);
                    tfx = -(nz * il); tfy = 0.f; tfz = nx * il;
                } else {
                    const float il = 1.f / sqrtf(ny * ny + nz * nz);
                    tfx = 0.f; tfy = nz * il; tfz = -(ny * il);
                }
                const float bfx = ny * tfz - nz * tfy, bfy = nz * tfx - nx * tfz, bfz = nx * tfy - ny * tfx;
                float X = 0.f, Y = 0.f;
                bool got = false;
                for (int q = 0; q < 4 && !got; q++) {
                    uint32_t rd[4];
                    pt_rand(pixel, s, b, 3 + q, P->seed, rd);
                    for (int k = 0; k < 2 && !got; k++) {
                        const float a = u01f(rd[2 * k]) * 2.f - 1.f, c = u01f(rd[2 * k + 1]) * 2.f - 1.f;
                        if (a * a + c * c < 1.f) { X = a; Y = c; got = true; }
                    }
                }
                const float Z = sqrtf(std::max(0.f, 1.f - X * X - Y * Y));
                float ndx = X * tfx + Y * bfx + Z * nx;
                float ndy = X * tfy + Y * bfy + Z * ny;
                float ndz = X * tfz + Y * bfz + Z * nz;
                const float dl = sqrtf(dot3f(ndx, ndy, ndz, ndx, ndy, ndz));
                ndx = ndx / dl; ndy = ndy / dl; ndz = ndz / dl;
                float t0 = tpf[0] * alb[0], t1 = tpf[1] * alb[1], t2 = tpf[2] * alb[2];
                double d0 = tpd[0] * alb[0], d1 = tpd[1] * alb[1], d2d = tpd[2] * alb[2];
                if (b >= P->rr_start) {
                    const float p = std::max(std::max(std::max(t0, t1), t2), 0.05f);
                    uint32_t rq[4];
                    pt_rand(pixel, s, b, 2, P->seed, rq);
                    if (u01f(rq[0]) >= p) break;
                    t0 = t0 / p; t1 = t1 / p; t2 = t2 / p;
                    d0 /= (double)p; d1 /= (double)p; d2d /= (double)p;
                }
                tpf[0] = t0; tpf[1] = t1; tpf[2] = t2;
                tpd[0] = d0; tpd[1] = d1; tpd[2] = d2d;
                ray.org[0] = ox; ray.org[1] = oy; ray.org[2] = oz; ray.tmin = 1e-4f;
                ray.dir[0] = ndx; ray.dir[1] = ndy; ray.dir[2] = ndz; ray.tmax = 1e30f;
            }
            for (int c = 0; c < 3; c++) acc[c] += L[c];
        }
        for (int c = 0; c < 3; c++) out_rgb[(size_t)ip * 3 + c] = acc[c] / spp;
        n_ext += ne;
        n_sha += ns;
    });
    if (ray_counts) { ray_counts[0] = n_ext.load(); ray_counts[1] = n_sha.load(); }
}

}  // extern "C"
