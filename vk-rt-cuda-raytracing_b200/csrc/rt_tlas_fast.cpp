// rt_tlas_fast.cpp -- cudaBVH_buildTLASFast: Morton LBVH over instance AABBs
// exported as a stackless BVH2 (reference: layer/cuda_bvh_backend.cu:257-389
// and :1620-1698).  The export format, the Morton code arithmetic, the
// stable 4 x 8-bit radix order, the median split and the single-instance
// leaves are kept so the node bytes match the reference's, with one
// difference: every skip pointer is the index after the node's subtree (the
// reference leaves the -2 placeholder on right descendants of left children,
// which ends a stackless walk early).  Host code: the layer calls it per
// frame on host AABBs and consumes host arrays.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/cuda_bvh_backend.h"

namespace {

uint32_t spread10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

uint32_t morton30(float x, float y, float z) {
    x = fminf(fmaxf(x * 1024.0f, 0.0f), 1023.0f);
    y = fminf(fmaxf(y * 1024.0f, 0.0f), 1023.0f);
    z = fminf(fmaxf(z * 1024.0f, 0.0f), 1023.0f);
    return spread10((uint32_t)x) * 4 + spread10((uint32_t)y) * 2 + spread10((uint32_t)z);
}

struct Node {
    float lo[3], hi[3];
    int left, right, first, count;
};

struct Lbvh {
    const float* sorted;
    std::vector<Node> nodes;
    int build(int s, int e) {
        Node nd;
        nd.left = nd.right = nd.first = nd.count = 0;
        for (int k = 0; k < 3; k++) { nd.lo[k] = 1e30f; nd.hi[k] = -1e30f; }
        const int cnt = e - s;
        if (cnt <= 1) {
            nd.first = s;
            nd.count = cnt;
            for (int i = s; i < e; i++)
                for (int k = 0; k < 3; k++) {
                    nd.lo[k] = fminf(nd.lo[k], sorted[i * 6 + k]);
                    nd.hi[k] = fmaxf(nd.hi[k], sorted[i * 6 + 3 + k]);
                }
            nodes.push_back(nd);
            return (int)nodes.size() - 1;
        }
        const int mid = s + cnt / 2;
        const int id = (int)nodes.size();
        nodes.push_back(nd);
        const int l = build(s, mid), r = build(mid, e);
        nodes[id].left = l;
        nodes[id].right = r;
        for (int k = 0; k < 3; k++) {
            nodes[id].lo[k] = fminf(nodes[l].lo[k], nodes[r].lo[k]);
            nodes[id].hi[k] = fmaxf(nodes[l].hi[k], nodes[r].hi[k]);
        }
        return id;
    }
};

}  // namespace

extern "C" int cudaBVH_buildTLASFast(const float* aabbs, int n, uint32_t** outNodes, int** outOrdered) {
    if (!aabbs || n <= 0 || !outNodes) return 0;
    *outNodes = nullptr;
    if (outOrdered) *outOrdered = nullptr;
    float smin[3] = {1e30f, 1e30f, 1e30f}, smax[3] = {-1e30f, -1e30f, -1e30f};
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            const float c = (aabbs[i * 6 + k] + aabbs[i * 6 + 3 + k]) * 0.5f;
            smin[k] = fminf(smin[k], c);
            smax[k] = fmaxf(smax[k], c);
        }
    float inv[3];
    for (int k = 0; k < 3; k++) inv[k] = (smax[k] - smin[k] > 1e-8f) ? 1.0f / (smax[k] - smin[k]) : 0.0f;
    std::vector<uint32_t> code(n);
    std::vector<int> idx(n), tmp(n);
    for (int i = 0; i < n; i++) {
        float c[3];
        for (int k = 0; k < 3; k++) c[k] = (aabbs[i * 6 + k] + aabbs[i * 6 + 3 + k]) * 0.5f;
        code[i] = morton30((c[0] - smin[0]) * inv[0], (c[1] - smin[1]) * inv[1], (c[2] - smin[2]) * inv[2]);
        idx[i] = i;
    }
    // stable LSD counting sort on 8-bit digits
    for (int sh = 0; sh < 32; sh += 8) {
        int start[257] = {0};
        for (int i = 0; i < n; i++) start[((code[idx[i]] >> sh) & 0xFFu) + 1]++;
        for (int b = 0; b < 256; b++) start[b + 1] += start[b];
        for (int i = 0; i < n; i++) tmp[start[(code[idx[i]] >> sh) & 0xFFu]++] = idx[i];
        idx.swap(tmp);
    }
    std::vector<float> sorted((size_t)n * 6);
    for (int i = 0; i < n; i++) memcpy(&sorted[(size_t)i * 6], aabbs + (size_t)idx[i] * 6, 24);
    Lbvh b;
    b.sorted = sorted.data();
    b.nodes.reserve((size_t)2 * n);
    b.build(0, n);
    // preorder export
    std::vector<int> order, stack{0};
    order.reserve(b.nodes.size());
    while (!stack.empty()) {
        const int i = stack.back();
        stack.pop_back();
        order.push_back(i);
        if (b.nodes[i].count == 0) {
            stack.push_back(b.nodes[i].right);
            stack.push_back(b.nodes[i].left);
        }
    }
    const int m = (int)order.size();
    std::vector<int> size(b.nodes.size(), 1);
    for (int k = m - 1; k >= 0; k--) {
        const Node& x = b.nodes[order[k]];
        if (x.count == 0) size[order[k]] = 1 + size[x.left] + size[x.right];
    }
    uint32_t* out = (uint32_t*)malloc((size_t)m * 8 * sizeof(uint32_t));
    if (!out) return 0;
    for (int k = 0; k < m; k++) {
        const Node& x = b.nodes[order[k]];
        uint32_t* p = out + (size_t)k * 8;
        memcpy(p, x.lo, 12);
        memcpy(p + 3, x.hi, 12);
        const int enc = x.count > 0 ? -((x.first << 3) | (x.count - 1)) - 2 : 0;
        const int skip = k + size[order[k]] < m ? k + size[order[k]] : -1;
        memcpy(p + 6, &enc, 4);
        memcpy(p + 7, &skip, 4);
    }
    *outNodes = out;
    if (outOrdered) {
        int* o = (int*)malloc((size_t)n * sizeof(int));
        if (o) memcpy(o, idx.data(), (size_t)n * sizeof(int));
        *outOrdered = o;
    }
    return m;
}
