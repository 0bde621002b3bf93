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
// Launch shape of the batched trace (the autotuner's choice).
using BatchShape = RtBatchTuning;
int launch_trace_multi(const Bvh8Device& b, const RtRay* rays, int n, const int* ray_off, const int* tri_off,
                       int nscenes, RtHit* hits, uint8_t* occ, int* work, int* status, const BatchShape& shape,
                       cudaStream_t s);

// A shared-wavefront segment: rays [first, next.first) of the launch are
// rays[0 ..] of this segment, traced from arena node `root`, results to out.
struct alignas(16) WaveSeg {
    const RtRay* rays;
    void* out;
    uint32_t first;
    uint32_t root;
    uint32_t pad[2];
};
enum { MODE_SINGLE = 0, MODE_BATCH = 1, MODE_WAVE = 2 };
int launch_trace_wave(const uint4* nodes, const float4* tris, const WaveSeg* segs, int nseg, int n, bool any,
                      int* work, int* status, int ctas_per_sm, cudaStream_t s);
void launch_rebase_nodes(const void* src, void* dst, int count, uint32_t node_off, uint32_t tri_off,
                         cudaStream_t s);

}  // namespace rtb
