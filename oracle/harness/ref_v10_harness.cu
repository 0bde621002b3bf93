// ref_v10_harness.cu -- drives the reference's own any-hit kernel traceShadow
// (v10_pipeline.cu:195-251) rebuilt for sm_100a.  Comparison arm only: this
// is how the in-run "rebuilt reference any-hit kernel" is timed.  The
// reference source is #included from where it lies (REF_V10_SOURCE, set by
// oracle/Makefile); its main() is renamed with -Dmain=ref_v10_main.  Nothing
// here changes the reference's kernels or builders; the harness builds the
// BVH the way main() does, converts ray layouts and launches.
#include REF_V10_SOURCE

#include <vector>

namespace {
struct RefV10 {
    int nt = 0, nc = 0, n4 = 0;
    int4* d_bvh4 = nullptr;
    float* d_v[9] = {nullptr};
    float* d_ray[9] = {nullptr};  // ox oy oz dx dy dz ix iy iz
    float* d_maxt = nullptr;
    int ray_cap = 0;
    unsigned long long* d_stats = nullptr;
};

// {float4 origin_tmin, float4 dir_tmax} -> the kernel's SoA arrays; the
// inverse direction is the plain 1/d of genShadow (v10_pipeline.cu:335) and
// the per-ray maximum distance is tmax.
__global__ void k_ray_soa(const float4* __restrict__ rays, int n, float* ox, float* oy, float* oz, float* dx,
                          float* dy, float* dz, float* ix, float* iy, float* iz, float* maxt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = rays[2 * i], b = rays[2 * i + 1];
    ox[i] = a.x; oy[i] = a.y; oz[i] = a.z;
    dx[i] = b.x; dy[i] = b.y; dz[i] = b.z;
    ix[i] = 1.f / b.x; iy[i] = 1.f / b.y; iz[i] = 1.f / b.z;
    maxt[i] = b.w;
}
}  // namespace

extern "C" {

int refv10_abi(void) { return 1; }

// BVH as main() builds it (v10_pipeline.cu:445-455): recursive 16-bin SAH
// with 4-triangle leaves (buildSAH), DFS reorder, collapse to BVH4,
// reorder, fp16 pack; top nodes into constant memory; triangles as SoA in
// leaf order.
void* refv10_build(const float* tris9, int n) {
    RefV10* h = new RefV10();
    h->nt = n;
    std::vector<Tri> tris(reinterpret_cast<const Tri*>(tris9), reinterpret_cast<const Tri*>(tris9) + n);
    std::vector<BN> nodes((size_t)n * 2);
    std::vector<int> tidx(n);
    for (int i = 0; i < n; i++) tidx[i] = i;
    int nc = 0;
    buildSAH(nodes.data(), tris.data(), tidx.data(), nc, 0, n, 0);
    h->nc = nc;
    std::vector<BN> ord(nc);
    std::vector<int> remap(nc);
    treeReorder(nodes.data(), nc, ord.data(), remap.data());
    std::vector<BVH4H> b4(nc), b4o;
    int n4 = 0;
    collapseRec(ord.data(), 0, b4.data(), &n4);
    b4o.resize(n4);
    std::vector<int> r4(n4);
    reorderBVH4(b4.data(), n4, b4o.data(), r4.data());
    std::vector<int4> gpu((size_t)n4 * 4);
    packBVH4GPU(b4o.data(), n4, gpu.data());
    h->n4 = n4;
    const int cn4 = n4 < CONST_BVH4 ? n4 : CONST_BVH4;
    cudaMemcpyToSymbol(c_bvh4, gpu.data(), cn4 * 4 * sizeof(int4));
    cudaMemcpyToSymbol(c_bvh4N, &cn4, 4);
    if (cudaMalloc(&h->d_bvh4, (size_t)n4 * 4 * sizeof(int4)) != cudaSuccess) return nullptr;
    cudaMemcpy(h->d_bvh4, gpu.data(), (size_t)n4 * 4 * sizeof(int4), cudaMemcpyHostToDevice);
    std::vector<float> soa(n);
    for (int c = 0; c < 9; c++) {
        for (int i = 0; i < n; i++) soa[i] = reinterpret_cast<const float*>(&tris[tidx[i]])[c];
        if (cudaMalloc(&h->d_v[c], (size_t)n * 4) != cudaSuccess) return nullptr;
        cudaMemcpy(h->d_v[c], soa.data(), (size_t)n * 4, cudaMemcpyHostToDevice);
    }
    if (cudaMalloc(&h->d_stats, 16) != cudaSuccess) return nullptr;
    return h;
}

int refv10_num_b4(void* hv) { return static_cast<RefV10*>(hv)->n4; }

// Converts n rays (device, 32 bytes each) into the kernel's input arrays;
// not part of the timed launch.
int refv10_set_rays(void* hv, const void* d_rays, int n, void* stream) {
    RefV10* h = static_cast<RefV10*>(hv);
    cudaStream_t s = (cudaStream_t)stream;
    if (n > h->ray_cap) {
        for (int c = 0; c < 9; c++) cudaFree(h->d_ray[c]);
        cudaFree(h->d_maxt);
        for (int c = 0; c < 9; c++)
            if (cudaMalloc(&h->d_ray[c], (size_t)n * 4) != cudaSuccess) return -1;
        if (cudaMalloc(&h->d_maxt, (size_t)n * 4) != cudaSuccess) return -1;
        h->ray_cap = n;
    }
    k_ray_soa<<<(n + 255) / 256, 256, 0, s>>>((const float4*)d_rays, n, h->d_ray[0], h->d_ray[1], h->d_ray[2],
                                              h->d_ray[3], h->d_ray[4], h->d_ray[5], h->d_ray[6], h->d_ray[7],
                                              h->d_ray[8], h->d_maxt);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// traceShadow launched as benchShadow does (v10_pipeline.cu:418-421):
// SMs x 4 persistent CTAs of 256 threads, 128 BVH4 nodes in shared memory.
// d_occ: one int per ray.
int refv10_trace_shadow(void* hv, void* d_occ, int n, int blocks, void* stream) {
    RefV10* h = static_cast<RefV10*>(hv);
    cudaStream_t s = (cudaStream_t)stream;
    if (n > h->ray_cap) return -1;
    const unsigned int z = 0;
    cudaMemcpyToSymbolAsync(g_rayCounter, &z, 4, 0, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(h->d_stats, 0, 16, s);
    const int smB = SMEM_BVH4_NODES * 4 * sizeof(int4);
    traceShadow<<<blocks, 256, smB, s>>>(h->d_bvh4, h->n4, SMEM_BVH4_NODES, h->d_v[0], h->d_v[1], h->d_v[2],
                                         h->d_v[3], h->d_v[4], h->d_v[5], h->d_v[6], h->d_v[7], h->d_v[8],
                                         h->d_ray[0], h->d_ray[1], h->d_ray[2], h->d_ray[3], h->d_ray[4],
                                         h->d_ray[5], h->d_ray[6], h->d_ray[7], h->d_ray[8], h->d_maxt,
                                         (int*)d_occ, n, h->d_stats);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

void refv10_destroy(void* hv) {
    RefV10* h = static_cast<RefV10*>(hv);
    if (!h) return;
    cudaFree(h->d_bvh4);
    for (int c = 0; c < 9; c++) {
        cudaFree(h->d_v[c]);
        cudaFree(h->d_ray[c]);
    }
    cudaFree(h->d_maxt);
    cudaFree(h->d_stats);
    delete h;
}

}  // extern "C"
