/* oracle.h -- CPU oracle for the ray-traversal hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls
 * this code; only tests/, __graft_entry__.smoke() and bench.py's CPU baseline
 * leg load it, to verify results against.
 *
 * What it restates (reference paths are relative to the reference project):
 *   - BVH2Builder::build/buildRec, binned SAH, layer/cuda_bvh_backend.cu:201-251
 *     (16 bins, leaf <= 3) and cuda_rt_v40.cu:790-840 (32 bins, maxLeaf knob);
 *   - collapseToB4 with fp16 round-to-nearest bounds, layer/cuda_bvh_backend.cu:391-418;
 *   - buildDFSBVH2 (stackless BVH2 with skip pointers), layer/cuda_bvh_backend.cu:456-522;
 *   - packed-triangle export, layer/cuda_bvh_backend.cu:716-735;
 *   - LBVHBuilder + cudaBVH_buildTLASFast, layer/cuda_bvh_backend.cu:257-389,1620-1698;
 *   - stackless traversal, layer/shaders/bvh2_stackless.comp:37-76, with the
 *     Moller-Trumbore arithmetic of layer/cuda_bvh_backend.cu:143-157;
 *   - two-level TLAS->BLAS traversal, layer/rt_ir_exec.cu:81-189;
 *   - Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11);
 *   - the engine's 8-wide compressed walk with its work counts, after the
 *     traceCWBVH scheme of cuda_rt_v37.cu:146-373 (node visits and triangle
 *     tests per ray, the basis of the algorithmic bytes per ray).
 *
 * Parity pinning: tests compare this restatement byte-for-byte against the
 * reference's own builder compiled from its sources into oracle/_ref/ and
 * against committed golden fixtures made from it (tests/golden/).
 */
#ifndef RT_ORACLE_H
#define RT_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float org[3]; float tmin; float dir[3]; float tmax; } OrcRay;   /* 32 B */
typedef struct { float t; int32_t prim; float u; float v; } OrcHit;              /* 16 B */

/* ---- builder restatement ---- */
void*  orc_build(const float* tris9, int n, int nbins, int max_leaf);
void   orc_free(void* h);
int    orc_num_bvh2(void* h);
int    orc_num_dfs(void* h);
const uint32_t* orc_dfs(void* h);          /* 8 u32 per node */
int    orc_num_packed(void* h);            /* vec4 count = 3 * ordered tris */
const float* orc_packed(void* h);          /* 12 floats per tri */
int    orc_num_bvh4(void* h);
const void* orc_bvh4(void* h);             /* 64 B per node */
const int*  orc_orig_idx(void* h);
void   orc_bounds(void* h, float* cx, float* cy, float* cz, float* extent);

int    orc_tlas_fast(const float* aabbs, int n, uint32_t** out_nodes, int** out_ordered);
void   orc_free_ptr(void* p);

/* ---- traversal restatement (closest hit, any hit) ---- */
/* Closest hit over a stackless BVH2 export + packed triangles.  prim is the
 * original primitive index stored in the packed triangle (p[9]).  Ties on t
 * are broken towards the lower prim.  stats (optional, 2 x u64 per ray):
 * inner-node visits and triangle tests. */
void orc_trace_closest_dfs(const uint32_t* dfs, int nnodes, const float* packed,
                           const OrcRay* rays, int nrays, OrcHit* hits,
                           int nthreads, uint64_t* stats);
void orc_trace_any_dfs(const uint32_t* dfs, int nnodes, const float* packed,
                       const OrcRay* rays, int nrays, uint8_t* occluded, int nthreads);
/* The engine's own 8-wide walk (nodes of 20 words, triangle records of 12
 * floats, as the library lays them out in device memory), restated with the
 * kernel's node-visit and triangle-test counts per ray (2 x u32 in counts).
 * any = 0: closest hit into hits; 1: occlusion flags into occluded.  niters:
 * node visits per round of the walk (the kernel's RTB_NODE_ITERS).  Returns
 * the number of rays whose walk left the arrays (0 for a valid tree). */
int orc_walk_bvh8(const uint32_t* nodes, int nnodes, const float* recs, int nrecs, const OrcRay* rays,
                  int nrays, int any, int niters, int sets, OrcHit* hits, uint8_t* occluded, uint32_t* counts,
                  int nthreads);
void orc_brute_closest(const float* tris9, int ntris, const OrcRay* rays, int nrays,
                       OrcHit* hits, int nthreads);
void orc_brute_any(const float* tris9, int ntris, const OrcRay* rays, int nrays,
                   uint8_t* occluded, int nthreads);

/* ---- two-level (instanced) traversal ----
 * blas_dfs/blas_packed: concatenated exports of every BLAS; per BLAS i its
 * node offset node_off[i] and packed-triangle offset tri_off[i] (in tris).
 * inst: 16 floats per instance: xform[12] row-major object->world, inv[12]
 * is computed by the caller into inv12 (12 floats per instance), blas index
 * in inst_blas[].  TLAS: stackless export over the instances (leaf index =
 * position in tlas_ordered[] -> instance id). */
void orc_trace_closest_two_level(const uint32_t* tlas, int tlas_nodes, const int* tlas_ordered,
                                 const float* inv12, const int* inst_blas, int ninst,
                                 const uint32_t* blas_dfs, const int* node_off,
                                 const float* blas_packed, const int* tri_off,
                                 const OrcRay* rays, int nrays, OrcHit* hits, int32_t* inst_out,
                                 int nthreads);
void orc_trace_any_two_level(const uint32_t* tlas, int tlas_nodes, const int* tlas_ordered,
                             const float* inv12, const int* inst_blas, int ninst,
                             const uint32_t* blas_dfs, const int* node_off,
                             const float* blas_packed, const int* tri_off,
                             const OrcRay* rays, int nrays, uint8_t* occluded, int nthreads);

/* ---- next-bounce ray generation (restates cudaBVH_generateRays) ----
 * kind 0: cosine-weighted diffuse, 1: shadow rays toward a square light.
 * Returns the number of rays written to out (and input indices to src). */
int orc_generate_rays(const float* tris9, int ntris, const OrcRay* rays, const OrcHit* hits, int n, int kind,
                      int count, uint32_t seed, float eps, float tmin, float tmax, const float* light_center,
                      float light_size, OrcRay* out, int32_t* src, int nthreads);

/* ---- Philox4x32-10 ---- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Recompute skip pointers of a stackless export in place (returns how many
 * changed, -1 if the array is not a well-formed preorder binary tree). */
int    orc_fix_skips(uint32_t* dfs, int n);

/* ---- FP64 path-tracing oracle (mirrors the wavefront path tracer) ---- */
typedef struct {
    const uint32_t* tlas; int tlas_nodes; const int* tlas_ordered;
    const float* inv12; const float* fwd12; const int* inst_blas; int ninst;
    const uint32_t* blas_dfs; const int* node_off; const float* blas_packed; const int* tri_off;
    const float* blas_tris9; const int* blas_tri_base; const int* blas_tri_count;
    const float* albedo3; const float* emission3;
} OrcPTScene;
typedef struct { int width, height, spp, max_bounces, rr_start; uint32_t seed; } OrcPTParams;
/* Radiance (double RGB) of the listed pixels; cam = the renderer's 14-float
 * camera basis; ray_counts (optional): extension and shadow rays traced. */
void orc_pt_pixels(const OrcPTScene* scene, const float* cam, const OrcPTParams* params, const int* pixels,
                   int npix, double* out_rgb, int nthreads, uint64_t* ray_counts);

/* ---- fp16 helpers (round to nearest even, as __float2half) ---- */
uint16_t orc_f2h_rn(float f);

#ifdef __cplusplus
}
#endif
#endif
