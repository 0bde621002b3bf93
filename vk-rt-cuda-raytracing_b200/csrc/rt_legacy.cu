// rt_legacy.cu -- ray generation and shading kernels behind the reference's
// original entry points (cudaBVH_tracePrimary, cudaBVH_traceDiffuse,
// cudaBVH_traceTo*).  Traversal itself always goes through the 8-wide
// closest-hit kernel (rt_trace.cu).
#include <cuda_fp16.h>

#include "rt_internal.h"
#include "rt_legacy.h"

namespace rtb {

// Square camera of layer/cuda_bvh_backend.cu:69-74: u, v = (p + 0.5)/side*2 - 1,
// d = (u, v, 1)/|(u, v, 1)|.  The reference used rsqrtf; 1/sqrtf keeps the
// direction reproducible on the host.
__global__ void k_gen_square(RtRay* __restrict__ rays, int side, float cx, float cy, float cz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= side * side) return;
    const int px = i % side, py = i / side;
    const float u = (px + 0.5f) / side * 2.f - 1.f;
    const float v = (py + 0.5f) / side * 2.f - 1.f;
    const float rl = 1.0f / sqrtf(u * u + v * v + 1.f);
    RtRay r;
    r.org[0] = cx; r.org[1] = cy; r.org[2] = cz; r.tmin = 0.f;
    r.dir[0] = u * rl; r.dir[1] = v * rl; r.dir[2] = rl; r.tmax = 1e30f;
    rays[i] = r;
}

// SoA host rays of cudaBVH_traceDiffuse (layer/cuda_bvh_backend.cu:1379-1497):
// accept t > 0, misses at 1e30.
__global__ void k_soa_rays(const float* __restrict__ soa, int n, RtRay* __restrict__ rays) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    RtRay r;
    r.org[0] = soa[i]; r.org[1] = soa[n + i]; r.org[2] = soa[2 * n + i]; r.tmin = 0.f;
    r.dir[0] = soa[3 * n + i]; r.dir[1] = soa[4 * n + i]; r.dir[2] = soa[5 * n + i]; r.tmax = 1e30f;
    rays[i] = r;
}

__global__ void k_hit_t(const RtHit* __restrict__ hits, int n, float* __restrict__ t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) t[i] = hits[i].prim >= 0 ? hits[i].t : 1e30f;
}

// Look-at camera of layer/cuda_bvh_backend.cu:856-868.
__global__ void k_gen_lookat(RtRay* __restrict__ rays, int w, int h, CamBasis c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    const int px = i % w, py = i / w;
    float u = ((float)px + 0.5f) / w * 2.f - 1.f;
    float v = ((float)py + 0.5f) / h * 2.f - 1.f;
    u *= (float)w / h * c.fov;
    v *= c.fov;
    float dx = c.fwd[0] + u * c.right[0] + v * c.up[0];
    float dy = c.fwd[1] + u * c.right[1] + v * c.up[1];
    float dz = c.fwd[2] + u * c.right[2] + v * c.up[2];
    const float rl = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
    RtRay r;
    r.org[0] = c.eye[0]; r.org[1] = c.eye[1]; r.org[2] = c.eye[2]; r.tmin = 0.f;
    r.dir[0] = dx * rl; r.dir[1] = dy * rl; r.dir[2] = dz * rl; r.tmax = 1e30f;
    rays[i] = r;
}

// Face-normal shading of layer/cuda_bvh_backend.cu:923-984 (sky gradient on a
// miss; ambient + key light + rim on a hit) into RGBA8/BGRA8/RGBA16F/RGBA32F.
__global__ void k_shade(const RtRay* __restrict__ rays, const RtHit* __restrict__ hits,
                        const float* __restrict__ tris9, int w, int h, void* __restrict__ out, int fmt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    const int py = i / w;
    const RtHit hh = hits[i];
    float rf, gf, bf;
    if (hh.prim < 0) {
        const float vv = (float)py / h;
        rf = (20.f + 10.f * (1.f - vv)) / 255.f;
        gf = (30.f + 20.f * (1.f - vv)) / 255.f;
        bf = (60.f + 100.f * vv) / 255.f;
    } else {
        const float* t = tris9 + (size_t)hh.prim * 9;
        const float e1x = t[3] - t[0], e1y = t[4] - t[1], e1z = t[5] - t[2];
        const float e2x = t[6] - t[0], e2y = t[7] - t[1], e2z = t[8] - t[2];
        float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
        const float nl = rsqrtf(nx * nx + ny * ny + nz * nz + 1e-20f);
        nx *= nl; ny *= nl; nz *= nl;
        const RtRay r = rays[i];
        if (nx * r.dir[0] + ny * r.dir[1] + nz * r.dir[2] > 0.f) { nx = -nx; ny = -ny; nz = -nz; }
        float lx = 0.5f, ly = 0.7f, lz = 0.5f;
        const float ll = rsqrtf(lx * lx + ly * ly + lz * lz);
        lx *= ll; ly *= ll; lz *= ll;
        const float ndotl = fmaxf(nx * lx + ny * ly + nz * lz, 0.f);
        const float ndotv = fabsf(-(nx * r.dir[0] + ny * r.dir[1] + nz * r.dir[2]));
        const float rim = 0.2f * powf(1.f - ndotv, 3.f);
        const float shade = fminf(0.15f + 0.65f * ndotl + rim, 1.f);
        rf = shade * 0.92f + 0.08f;
        gf = shade * 0.88f + 0.07f;
        bf = shade * 0.82f + 0.06f;
    }
    if (fmt == 3) {
        reinterpret_cast<float4*>(out)[i] = make_float4(rf, gf, bf, 1.f);
    } else if (fmt == 2) {
        __half* o = reinterpret_cast<__half*>(out) + (size_t)i * 4;
        o[0] = __float2half(rf); o[1] = __float2half(gf); o[2] = __float2half(bf); o[3] = __float2half(1.f);
    } else {
        const uint32_t R = (uint32_t)(uint8_t)(rf * 255.f), G = (uint32_t)(uint8_t)(gf * 255.f),
                       B = (uint32_t)(uint8_t)(bf * 255.f);
        reinterpret_cast<uint32_t*>(out)[i] =
            fmt == 1 ? (255u << 24) | (R << 16) | (G << 8) | B : (255u << 24) | (B << 16) | (G << 8) | R;
    }
}

void launch_gen_square(RtRay* rays, int side, float cx, float cy, float cz, cudaStream_t s) {
    const int n = side * side;
    k_gen_square<<<(n + 255) / 256, 256, 0, s>>>(rays, side, cx, cy, cz);
}
void launch_soa_rays(const float* soa, int n, RtRay* rays, cudaStream_t s) {
    k_soa_rays<<<(n + 255) / 256, 256, 0, s>>>(soa, n, rays);
}
void launch_hit_t(const RtHit* hits, int n, float* t, cudaStream_t s) {
    k_hit_t<<<(n + 255) / 256, 256, 0, s>>>(hits, n, t);
}
void launch_gen_lookat(RtRay* rays, int w, int h, const CamBasis& c, cudaStream_t s) {
    k_gen_lookat<<<(w * h + 255) / 256, 256, 0, s>>>(rays, w, h, c);
}
void launch_shade(const RtRay* rays, const RtHit* hits, const float* tris9, int w, int h, void* out, int fmt,
                  cudaStream_t s) {
    k_shade<<<(w * h + 255) / 256, 256, 0, s>>>(rays, hits, tris9, w, h, out, fmt);
}

}  // namespace rtb
