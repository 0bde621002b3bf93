// rt_legacy.h -- launchers for the reference-shaped entry points.
#pragma once
#include <cuda_runtime.h>

#include "../../include/rt_b200.h"

namespace rtb {

struct CamBasis {
    float eye[3], fwd[3], right[3], up[3];
    float fov;
};

void launch_gen_square(RtRay* rays, int side, float cx, float cy, float cz, cudaStream_t s);
void launch_soa_rays(const float* soa, int n, RtRay* rays, cudaStream_t s);
void launch_hit_t(const RtHit* hits, int n, float* t, cudaStream_t s);
void launch_gen_lookat(RtRay* rays, int w, int h, const CamBasis& c, cudaStream_t s);
void launch_shade(const RtRay* rays, const RtHit* hits, const float* tris9, int w, int h, void* out, int fmt,
                  cudaStream_t s);

struct Bvh8Device;
int launch_trace_blas(const Bvh8Device& b, const RtRay* rays, int n, RtHit* hits, uint8_t* occ,
                      uint32_t* counts, int* work, int* status, cudaStream_t s);
int launch_trace_multi(const Bvh8Device& b, const RtRay* rays, int n, const int* ray_off, const int* tri_off,
                       int nscenes, RtHit* hits, uint8_t* occ, int* work, int* status, int ctas_per_sm,
                       int node_iters, cudaStream_t s);

}  // namespace rtb
