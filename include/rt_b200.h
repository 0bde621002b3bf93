/* rt_b200.h -- extension C-ABI of the B200 ray traversal engine.
 *
 * The reference's C-ABI (cuda_bvh_backend.h) has no closest-hit call that
 * returns primitive ids and barycentrics, no any-hit call, no instanced
 * (TLAS) trace, and no stream or batch parameters (reference
 * layer/cuda_bvh_backend.h:26-40 traces with hit distance only, on the
 * default stream).  These entry points fill those gaps with the same
 * conventions: opaque handles, plain pointers and sizes, int status (0 ok,
 * negative error; rtGetLastError() explains the last one on this thread).
 * `stream` is a cudaStream_t passed as void* (NULL = default stream); every
 * device-pointer call is asynchronous on that stream.
 */
#ifndef RT_B200_H
#define RT_B200_H

#include <stdint.h>

#include "cuda_bvh_backend.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A ray: origin, tmin, direction (need not be unit length), tmax.  32 bytes,
 * 16-byte aligned.  Hits are accepted for tmin < t < tmax.  This is the
 * reference prototypes' Ray {float4 origin_tmin, float4 dir_tmax}
 * (cuda_rt_v40.cu:30). */
typedef struct {
    float org[3];
    float tmin;
    float dir[3];
    float tmax;
} RtRay;

/* Closest-hit record, 16 bytes: t (+inf on a miss), the input index of the
 * hit primitive (-1 on a miss), Moller-Trumbore barycentrics.  Equal t is
 * resolved toward the lower (instance, primitive) id. */
typedef struct {
    float t;
    int32_t prim;
    float u;
    float v;
} RtHit;

/* Status codes. */
#define RT_OK 0
#define RT_ERR_INVALID (-1)   /* bad argument */
#define RT_ERR_CUDA (-2)      /* CUDA runtime error */
#define RT_ERR_NOMEM (-3)     /* device allocation failed */
#define RT_ERR_STACK (-4)     /* traversal stack overflow (never silent) */
#define RT_ERR_TIMEOUT (-5)   /* a bounded wait ran out */
#define RT_ERR_CAPACITY (-6)  /* admission / size limit */

/* Message of the last failure on the calling thread ("" if none). */
const char* rtGetLastError(void);

/* Build from triangles already in device memory (9 floats each); the build
 * runs on `stream` and the call returns once the structure is ready.
 * NULL on failure. */
CudaBVH_t cudaBVH_buildDevice(const CudaTri* d_tris, int numTris, void* stream);

/* Closest hit of n rays (device pointers).  Returns RT_OK or an error. */
int cudaBVH_traceClosest(CudaBVH_t bvh, const RtRay* d_rays, int n, RtHit* d_hits, void* stream);

/* Any hit (occlusion) of n rays: d_occluded[i] = 1 if some primitive is hit
 * with tmin < t < tmax, else 0. */
int cudaBVH_traceAny(CudaBVH_t bvh, const RtRay* d_rays, int n, uint8_t* d_occluded, void* stream);

/* ---- Next-bounce rays made on the device (the reference's genAndCompact,
 * multi_bounce.cu:281-362) ----
 * From a closest-hit batch traced on this BVH: for every input ray i whose
 * hit names one of this BVH's triangles, the hit point p = o + t d and the
 * triangle's geometric normal n turned to face the ray; the new ray starts
 * at p + eps n and goes
 *   RT_GEN_DIFFUSE: in a cosine-weighted direction about n (Malley's method:
 *     the first of eight Philox uniform points of [-1,1)^2 that lies in the
 *     unit disk, lifted to the hemisphere), over [tmin, tmax];
 *   RT_GEN_SHADOW: toward a uniform point of a light_size x light_size square
 *     parallel to xz centred at light_center, over [tmin, 0.9999 * distance].
 * Misses are dropped and the survivors compacted in input order (warp ballot
 * and block scan; deterministic).  count == 0: one ray per hit, output k from
 * the k-th hit; count > 0: exactly count rays, output k from the
 * (k mod hits)-th hit (none when there are no hits).  Random numbers: Philox
 * key (seed, 3) diffuse / (seed, 4) shadow, counter (k, block, 0, 0).  All
 * arithmetic is correctly rounded single precision without contraction, so
 * a CPU restatement reproduces every bit.  d_out holds n rays (count == 0)
 * or count rays; d_src (optional) receives each output's input index;
 * *d_count (device) the number of rays written.  Stream-ordered; scratch
 * comes from the library's stream-ordered pool.  The reference's version
 * uses PCG, rsqrtf and sin/cos, and an atomic per block (output order
 * varies run to run). */
#define RT_GEN_DIFFUSE 0
#define RT_GEN_SHADOW 1
typedef struct {
    int kind;               /* RT_GEN_DIFFUSE or RT_GEN_SHADOW */
    int count;              /* 0: one ray per hit; > 0: exactly this many */
    uint32_t seed;          /* Philox key word 0 */
    float eps;              /* origin offset along the facing normal (0.001 in the reference) */
    float tmin, tmax;       /* diffuse: the new rays' interval; shadow: tmin only */
    float light_center[3];  /* shadow rays: centre of the square light */
    float light_size;       /* shadow rays: side of the square light */
} RtRayGen;
int cudaBVH_generateRays(CudaBVH_t bvh, const RtRay* d_rays, const RtHit* d_hits, int n, const RtRayGen* gen,
                         RtRay* d_out, int32_t* d_src, int* d_count, void* stream);

/* Traversal status of the device-pointer calls on this handle.  The trace
 * calls above return as soon as the kernel is queued, so a stack overflow
 * inside it (RT_ERR_STACK: the BVH is deeper than the 64-entry traversal
 * stack; never silent) is recorded in the handle's status word instead.
 * This call waits for `stream`, reads the word, clears it and returns
 * RT_OK or RT_ERR_STACK (or RT_ERR_CUDA).  The word is shared by every call
 * on the handle since the last check, from any thread or stream.  The
 * reference has no counterpart (its trace calls only print CUDA errors,
 * layer/cuda_bvh_backend.cu:25). */
int cudaBVH_getStatus(CudaBVH_t bvh, void* stream);

/* The same two calls on host buffers: copies in, traces, copies out and
 * waits.  Staging buffers are owned by the handle. */
int cudaBVH_traceClosestHost(CudaBVH_t bvh, const RtRay* h_rays, int n, RtHit* h_hits);
int cudaBVH_traceAnyHost(CudaBVH_t bvh, const RtRay* h_rays, int n, uint8_t* h_occluded);

/* The same host-buffer traces over several replicas of one scene, one
 * handle per GPU (each built with its device current): the n rays split into
 * `count` contiguous blocks, as even as possible in handle order, and each
 * block runs through its handle's host pipeline on its own device from its
 * own host thread, so the GPUs' copy engines and SMs work at once.  Returns
 * when every result is in host memory; the first failing block's code, with
 * the replica's index in rtGetLastError().  At most 64 handles.  No
 * counterpart in the reference (one device per process there). */
int cudaBVH_traceClosestHostMulti(const CudaBVH_t* bvhs, int count, const RtRay* h_rays, int n, RtHit* h_hits);
int cudaBVH_traceAnyHostMulti(const CudaBVH_t* bvhs, int count, const RtRay* h_rays, int n, uint8_t* h_occluded);

/* Closest hit of up to 65,536 host rays without allocating any memory.
 * No counterpart in the reference.  For callers that must not allocate while
 * they trace: a Vulkan layer tracing on the application's render thread (a
 * cudaMalloc there can synchronise the device and stall the frame, and the
 * application owns the memory budget), real-time callers that cannot afford
 * the implicit synchronisation of cudaMalloc/cudaFree, and code running under
 * a fixed memory cap.  Rays and hits are staged in one fixed device array
 * compiled into the library (about 3 MiB, held by every GPU that loads the
 * library until exit); more than 65,536 rays -> RT_ERR_CAPACITY.  The first
 * call on each device looks up that array's device address (make it before
 * any stream capture).  All calls share the array: calls whose GPU work
 * overlaps corrupt each other's rays and hits, so serialise them.  Waits
 * for the result on `stream`.  Same results as cudaBVH_traceClosestHost. */
int cudaBVH_traceClosestHostNoAlloc(CudaBVH_t bvh, const RtRay* h_rays, int n, RtHit* h_hits, void* stream);

/* Host-side structural check of the built acceleration structure (child
 * indices, triangle ranges, depth within the traversal stack, every
 * triangle referenced once).  RT_OK or RT_ERR_INVALID.  Setting the
 * environment variable RTB200_VALIDATE=1 runs it inside every build. */
int cudaBVH_validate(CudaBVH_t bvh);

/* Build statistics. */
typedef struct {
    int num_tris;
    int num_bvh2_nodes;     /* binary nodes created by the SAH builder */
    int num_nodes;          /* compressed 8-wide nodes */
    int depth;              /* 8-wide levels */
    int max_leaf;
    int bins;
    float build_ms;         /* device time of the build kernels: the triangle
                               boxes and the build's one graph launch (the
                               host's graph capture and instantiation are not
                               in it); with RTB200_BUILD=host, the span of the
                               host-driven launches on the stream */
    float sah_cost;         /* SAH cost of the binary tree, normalised by root area */
    uint64_t node_bytes;    /* bytes of the 8-wide nodes */
    uint64_t tri_bytes;     /* bytes of the triangle records */
} RtBuildStats;
int cudaBVH_getBuildStats(CudaBVH_t bvh, RtBuildStats* out);

/* Device arrays of the 8-wide layout (80-byte nodes, 48-byte triangles),
 * borrowed, valid until destroy. */
int cudaBVH_getDeviceLayout(CudaBVH_t bvh, const void** d_nodes, int* num_nodes, const void** d_tris,
                            int* num_tris);

/* Closest hit with per-ray work counters (d_counts: 2 u32 per ray: nodes
 * fetched, triangles tested).  Same results as cudaBVH_traceClosest; used to
 * derive the algorithmic bytes per ray.  any != 0 counts the any-hit walk. */
int cudaBVH_traceCounters(CudaBVH_t bvh, const RtRay* d_rays, int n, int any, uint32_t* d_counts,
                          void* stream);

/* Test hook, no counterpart in the reference: after `after` more device
 * allocations by the library (handle buffers, staging, build scratch), every
 * further one fails as if the device were out of memory, until the hook is
 * called again; after < 0 turns it off.  The failing call returns
 * RT_ERR_NOMEM (or NULL for a build) with the reason in rtGetLastError(),
 * and the library stays usable.  Process-wide. */
int rtDebug_failAllocations(int after);

/* Inspection helper, no counterpart in the reference: the scene groups
 * rtBatch_build would use for these offsets (RTB200_BATCH_GROUPS honoured).
 * Writes the group count + 1 boundaries (scene indices, first 0, last
 * num_scenes) to out_bounds, which holds max_groups + 1 entries, and returns
 * the group count; RT_ERR_INVALID on bad arguments.  Host only: no device
 * work. */
int rtDebug_batchGroups(const int* tri_offsets, int num_scenes, int* out_bounds, int max_groups);

/* Measurement helper, no counterpart in the reference: read bandwidth of
 * this GPU in GB/s, streaming a `bytes` buffer (allocated and freed by the
 * call) `reps` times in one launch with 16-byte loads cached in L2 only,
 * timed with events after two warm-up passes.  A buffer well under the 126 MB L2 gives
 * the L2 read bandwidth that bounds traversal of an L2-resident BVH; one
 * far above it gives the HBM read bandwidth.  Changes no device setting. */
int rtProbe_readBandwidth(uint64_t bytes, int reps, float* out_gbs);

/* ---- Ray regrouping (the reference's Morton sort of ray origins before
 * tracing: CUB radix sort in cuda_rt_v40.cu:94-124,1226-1239, and a host
 * radix sort in its per-call path, layer/cuda_bvh_backend.cu:1387-1433) ----
 * d_out[k] = d_in[perm[k]] ordered by a key per ray: RT_REGROUP_MORTON, the
 * 30-bit Morton code of the origin in box6 = {lo x, y, z, hi x, y, z} (10
 * bits per axis, as the reference); RT_REGROUP_OCTANT_MORTON, the direction
 * octant above the top 29 bits of that code.  key_bits 16 sorts by the
 * key's top 16 bits only (2 passes of the radix sort instead of 4).  The
 * sort is stable (equal keys keep their input order) and runs on the device
 * with the library's own radix sort; d_perm (optional) receives the source
 * index of every output ray.  d_in and d_out must not overlap. */
#define RT_REGROUP_MORTON 0
#define RT_REGROUP_OCTANT_MORTON 1
int rtRays_regroup(const RtRay* d_in, int n, const float* box6, int kind, int key_bits, RtRay* d_out,
                   int32_t* d_perm, void* stream);

/* ---------------- instanced scenes (TLAS over BLASes) ---------------- */
typedef struct CudaTLASHandle* CudaTLAS_t;

/* One instance: row-major 3x4 object->world transform, the index of its
 * BLAS in the array given to cudaTLAS_build, and a user id.  64 bytes.
 * The layer's packing of VkAccelerationStructureInstanceKHR
 * (layer/VkLayer_CudaRT.cpp:4517-4558) carries the same fields. */
typedef struct {
    float xform[12];
    int32_t blas;
    uint32_t mask;
    uint32_t custom;
    uint32_t pad;
} RtInstance;

/* Builds the top level over world-space instance boxes on the GPU.  The
 * BLAS handles must outlive the TLAS.  NULL on failure. */
CudaTLAS_t cudaTLAS_build(const CudaBVH_t* blas, int numBlas, const RtInstance* instances, int numInstances);
void cudaTLAS_destroy(CudaTLAS_t tlas);

/* Per-frame instance update (replaces the layer's TLAS rebuild in
 * processPendingTLAS, layer/VkLayer_CudaRT.cpp:3418, paced by
 * CUDA_RT_TLAS_EVERY_N): new transforms and BLAS choices for the same number
 * of instances (over the BLAS array given to cudaTLAS_build); the top level
 * is rebuilt in place, the BLASes are untouched, and traces afterwards equal
 * those of a TLAS built with the new instances.  Waits for the device first
 * (traces in flight finish on the old instances).  On failure the TLAS keeps
 * its previous instances.  A path tracer created on the TLAS reloads the
 * transforms, BLAS choices and light areas at its next rtPT_render.  Safe
 * against traces and renders of the same TLAS on other threads: each takes
 * the TLAS's lock while it launches, so it runs wholly on the old or wholly
 * on the new instances. */
int cudaTLAS_setTransforms(CudaTLAS_t tlas, const RtInstance* instances, int numInstances);

/* Closest hit over all instances: d_hits[i].prim is the primitive index in
 * the hit instance's BLAS, d_inst[i] the instance index (-1 on a miss; may
 * be NULL).  Rays are transformed by the inverse instance transform without
 * renormalisation, so t is in world units. */
int cudaTLAS_traceClosest(CudaTLAS_t tlas, const RtRay* d_rays, int n, RtHit* d_hits, int32_t* d_inst,
                          void* stream);
int cudaTLAS_traceAny(CudaTLAS_t tlas, const RtRay* d_rays, int n, uint8_t* d_occluded, void* stream);

/* Status word of the TLAS's device-pointer traces, as cudaBVH_getStatus. */
int cudaTLAS_getStatus(CudaTLAS_t tlas, void* stream);

/* Inverse transforms (12 floats per instance) the TLAS uses, host copy. */
int cudaTLAS_getInverseTransforms(CudaTLAS_t tlas, float* out, int numInstances);

/* ---------------- batched scenes ----------------
 * Many independent scenes built in one multi-scene SAH build (every build
 * stage is one launch for all scenes, all of it one CUDA graph) and traced
 * by one persistent work-stealing launch.  A batch of 8M triangles or more
 * is built as two groups of whole scenes, one graph launch each, so the
 * first group builds while the second group's triangles are uploaded
 * (page-locked input: both copies queued at once); the groups merge into
 * the one layout below.  RTB200_BATCH_GROUPS=<g> sets the group count.  Triangles of scene i are tri_offsets[i] ..
 * tri_offsets[i+1]-1 of h_tris; rays of scene i are d_ray_offsets[i] ..
 * d_ray_offsets[i+1]-1 (device array, num_scenes+1 entries), at most
 * 65,535 scenes per batch.  Reported primitive ids are relative to their
 * scene. */
typedef struct RtBatchHandle* RtBatch_t;
RtBatch_t rtBatch_build(const CudaTri* h_tris, const int* tri_offsets, int num_scenes, void* stream);
/* rtBatch_build runs each group's whole build (SAH levels, small and warp
 * subtrees, 8-wide collapse) as ONE CUDA graph launch: both level loops are
 * conditional WHILE nodes whose counts stay on the device.  flags
 * RT_BATCH_BUILD_HOST_LOOP instead drives the same kernels from the host,
 * level by level (the single-scene builder's loop), over the same groups.
 * Both give the same layout, byte for byte. */
#define RT_BATCH_BUILD_HOST_LOOP 1
RtBatch_t rtBatch_buildEx(const CudaTri* h_tris, const int* tri_offsets, int num_scenes, int flags, void* stream);
void rtBatch_destroy(RtBatch_t batch);
int rtBatch_traceClosest(RtBatch_t batch, const RtRay* d_rays, const int* d_ray_offsets, int n, RtHit* d_hits,
                         void* stream);
int rtBatch_traceAny(RtBatch_t batch, const RtRay* d_rays, const int* d_ray_offsets, int n, uint8_t* d_occluded,
                     void* stream);
/* Same trace, replayed from a CUDA graph captured on the first call with
 * these arguments (re-captured when the arguments or the tuning change).
 * any != 0: d_out is uint8_t occlusion, else RtHit. */
int rtBatch_traceGraph(RtBatch_t batch, const RtRay* d_rays, const int* d_ray_offsets, int n, void* d_out, int any,
                       void* stream);
/* Launch shape of the batched trace. */
typedef struct {
    int warps_per_sm;   /* persistent worker warps per SM (8..32 at 128 threads per CTA) */
    int node_iters;     /* node visits per lane between pooled triangle phases (2..4) */
    int block;          /* threads per CTA: 64, 128 or 256 */
    int shared_stack;   /* traversal stack entries per ray kept in shared memory: 4, 8 or 12 */
} RtBatchTuning;
/* Autotuner: times the batch's closest-hit trace over the launch shape, one
 * dimension at a time from the default (worker warps per SM {8, 16, 24, 32},
 * node visits per iteration {2, 3, 4}, threads per CTA {64, 128, 256}, shared
 * stack entries {4, 8, 12}), keeping the fastest value of each before the
 * next.  With the environment variable RTB200_TUNE_CACHE=<file> the choice is
 * stored and reused.  out_ctas_per_sm reports the worker count as CTAs of
 * 128 threads; rtBatch_getTuning gives the whole shape. */
int rtBatch_autotune(RtBatch_t batch, const RtRay* d_rays, const int* d_ray_offsets, int n, RtHit* d_hits,
                     void* stream, int* out_ctas_per_sm, int* out_node_iters);
/* Worker count as CTAs of 128 threads per SM (1..8) and node visits (1..4);
 * block and shared stack keep their values. */
int rtBatch_setTuning(RtBatch_t batch, int ctas_per_sm, int node_iters);
int rtBatch_setTuningEx(RtBatch_t batch, const RtBatchTuning* tuning);
int rtBatch_getTuning(RtBatch_t batch, RtBatchTuning* out);
/* build_ms: device time of the build kernels, as RtBuildStats.build_ms. */
/* build_ms: device time of the build kernels (every group's triangle boxes
 * and graph launch, and the merge), as RtBuildStats.build_ms. */
int rtBatch_getInfo(RtBatch_t batch, int* num_scenes, int* num_nodes, float* build_ms);
/* Device arrays of the batch's 8-wide layout (scene i's root is node i;
 * triangle records carry scene-relative primitive ids), borrowed, valid
 * until destroy. */
int rtBatch_getDeviceLayout(RtBatch_t batch, const void** d_nodes, int* num_nodes, const void** d_tris,
                            int* num_tris);

/* ---------------- wavefront path tracer ----------------
 * Lambertian scene over a TLAS: per-instance albedo and emission; emission
 * counted on camera hits; next-event estimation toward one emissive triangle
 * (area-proportional choice, exact integer CDF; two-sided emitters);
 * cosine-weighted bounces; Russian roulette from bounce rr_start with
 * p = max(max throughput component, 0.05); black environment.  Philox4x32-10
 * keyed by (seed, pixel, sample, bounce), so a pixel's value does not depend
 * on how paths are scheduled.  Output: W*H*3 floats (RGB), row-major. */
typedef struct {
    float albedo[3];
    float emission[3];
} RtMaterial;

typedef struct {
    float eye[3];
    float target[3];
    float up[3];
    float vfov_deg;
} RtCamera;

typedef struct {
    int width, height, spp;
    int max_bounces;  /* path vertices, 1..16 */
    int rr_start;     /* first bounce with Russian roulette */
    uint32_t seed;
} RtPTParams;

typedef struct {
    uint64_t extension_rays;  /* closest-hit rays traced by the last render */
    uint64_t shadow_rays;     /* any-hit rays traced by the last render */
    int light_tris;
    double light_area;
} RtPTStats;

typedef struct RtPathTracerHandle* RtPathTracer_t;

/* materials[i] and instances[i] describe TLAS instance i (the same records
 * given to cudaTLAS_build).  The TLAS and its BLASes must outlive the path
 * tracer.  NULL on failure. */
RtPathTracer_t rtPT_create(CudaTLAS_t tlas, const RtMaterial* materials, int numMaterials,
                           const RtInstance* instances);
/* Renders into d_rgb (device, W*H*3 floats) on `stream`; path state buffers
 * are owned by the handle and grow to W*H*spp paths. */
int rtPT_render(RtPathTracer_t pt, const RtCamera* cam, const RtPTParams* params, float* d_rgb, void* stream);
int rtPT_getStats(RtPathTracer_t pt, RtPTStats* out);
/* Regroups each bounce's extension rays (after the camera rays) with
 * rtRays_regroup's key (kind, key_bits 16 or 32; 0 = off, the default)
 * before they are traced.  Paths are independent, so the image is the same
 * either way; only the order the rays are traced in changes. */
int rtPT_setRegroup(RtPathTracer_t pt, int kind, int key_bits);
/* Wavefront queue capacity: the frame's W*H*spp paths are traced in slices
 * of at most `paths` paths (contiguous path ids, each slice through all its
 * bounces before the next starts); 0 = the whole frame in one slice (the
 * default).  Queues take about 150 bytes per path of capacity.  The image
 * does not depend on it: every path keeps its own radiance slot. */
int rtPT_setQueueCapacity(RtPathTracer_t pt, int64_t paths);
/* Times renders of this frame with the whole frame, 1/2, 1/4 and 1/8 of it
 * per slice (slices that would not fill the GPU are skipped), keeps the
 * fastest capacity and returns it in *out_paths (0 = whole frame).  Renders
 * into d_rgb. */
int rtPT_autotune(RtPathTracer_t pt, const RtCamera* cam, const RtPTParams* params, float* d_rgb, void* stream,
                  int64_t* out_paths);
void rtPT_destroy(RtPathTracer_t pt);
/* The fp32 camera basis the renderer uses: eye[3], forward[3], right[3],
 * up[3], tan(vfov/2), aspect (14 floats). */
int rtPT_cameraBasis(const RtCamera* cam, int width, int height, float* out14);

/* ---- Geometry from the application's buffers, refit, blobs ---------------
 * The callers on either side of the build: the reference layer reads every
 * BLAS's vertex and index buffers back to the host and rebuilds a triangle
 * soup there
 * (layer/VkLayer_CudaRT.cpp:2961-2981, 3087-3125); refit and a versioned BVH
 * blob have no counterpart in the reference. */
#define RT_VERTEX_FLOAT3 0   /* 3 x fp32 per vertex (VK_FORMAT_R32G32B32_SFLOAT) */
#define RT_VERTEX_HALF3 1    /* 3 x fp16 per vertex (R16G16B16[A16]_SFLOAT) */
#define RT_INDEX_NONE 0      /* triangle p uses vertices 3p, 3p+1, 3p+2 */
#define RT_INDEX_UINT16 1
#define RT_INDEX_UINT32 2
typedef struct {
    const void* d_vertices;   /* device address of vertex 0 */
    uint64_t vertex_stride;   /* bytes from one vertex to the next */
    int vertex_format;        /* RT_VERTEX_* */
    int max_vertex;           /* highest vertex index the triangles may use */
    const void* d_indices;    /* device index buffer, or NULL with RT_INDEX_NONE */
    int index_type;           /* RT_INDEX_* */
    int num_triangles;
    const float* transform;   /* host 3x4 row-major object transform, or NULL */
} RtGeometry;

/* Builds a BLAS from num_geoms geometries (triangles of all geometries in
 * order; primitive ids count across them).  Triangles are gathered on the
 * device; an index above max_vertex is an error, never a read past the
 * buffer.  NULL on failure. */
CudaBVH_t cudaBVH_buildGeometries(const RtGeometry* geoms, int num_geoms, void* stream);

/* Refit after the vertices moved: same triangle count and order, new
 * positions (device CudaTri array, or the geometries as above).  Keeps the
 * tree's topology and recomputes every box; a TLAS over this BLAS must be
 * rebuilt afterwards (its instance boxes change).  Must not overlap traces
 * of the same handle.  RT_OK or an error. */
int cudaBVH_refit(CudaBVH_t bvh, const CudaTri* d_tris, void* stream);
int cudaBVH_refitGeometries(CudaBVH_t bvh, const RtGeometry* geoms, int num_geoms, void* stream);

/* Versioned, checksummed host blob of a BLAS (input triangles, binary BVH,
 * 8-wide nodes, triangle records).  buf == NULL: *size receives the bytes
 * needed.  RT_ERR_CAPACITY if capacity is too small. */
int cudaBVH_serialize(CudaBVH_t bvh, void* buf, uint64_t capacity, uint64_t* size);
/* Loads a blob (no rebuild): NULL with an error for a wrong magic or
 * version, a truncated or corrupted blob (checksum), or a structure that
 * fails validation. */
CudaBVH_t cudaBVH_deserialize(const void* buf, uint64_t size);

/* ---- Served form: a request loop over scenes resident in HBM ------------
 * No counterpart in the reference (its layer calls one synchronous trace per
 * ray batch, layer/cuda_bvh_backend.cu:526-598).  Scenes are copied into one
 * device arena; clients submit requests from any thread; a scheduler thread
 * admits host-buffer requests by footprint (rays + results) under the HBM
 * budget, packs the rays of admitted requests (oldest first, in chunks) into
 * shared wavefronts traced by one persistent launch per hit kind, keeps up
 * to max_waves wavefronts in flight, and copies each chunk's results back
 * as soon as it is traced.  A request's results are bit-identical to
 * cudaBVH_traceClosest / cudaBVH_traceAny of the same rays on the scene's
 * BVH, whatever else is in flight.  Host buffers should be pinned (page-
 * locked) for the copies to overlap; they must stay valid until the request
 * is waited for.  Every ticket must be waited for once (that frees it). */
typedef struct RtServerHandle* RtServer_t;
typedef struct {
    uint64_t hbm_budget_bytes; /* resident scenes + admitted request buffers; 0 = 120 GiB */
    uint64_t pool_bytes;       /* device staging pool for host-buffer requests; 0 = 4 GiB */
    int max_inflight;          /* requests admitted at once; 0 = 256 */
    int wave_rays;             /* rays per shared wavefront; 0 = 4 Mi */
    int chunk_rays;            /* rays per chunk of a request; 0 = 1 Mi */
    int max_waves;             /* wavefronts in flight, each on its own stream (1..8); 0 = 2 */
    int prefetch_rays;         /* copied rays waiting for a wavefront, at most; 0 = 2 * wave_rays */
} RtServerConfig;
typedef struct {
    double submit_us, admit_us, done_us; /* steady clock, microseconds since rtServer_create */
    int status;                          /* RT_OK, RT_ERR_STACK or RT_ERR_CUDA */
    int waves;                           /* wavefronts the request's chunks were traced in */
} RtRequestInfo;
typedef struct {
    uint64_t requests_done, rays_done, waves;
    uint64_t resident_bytes, pool_bytes, peak_pool_used;
    int num_scenes;
} RtServerStats;

/* cfg may be NULL (all defaults).  The server runs on the current device. */
RtServer_t rtServer_create(const RtServerConfig* cfg);
/* Copies the BVH into the resident arena (the handle may be destroyed
 * afterwards).  Returns the scene id (>= 0) or RT_ERR_CAPACITY when the
 * budget would be exceeded, another error code otherwise.  Waits until no
 * wavefront is in flight. */
int rtServer_addScene(RtServer_t s, CudaBVH_t bvh);
/* Host-buffer request: n rays in h_rays, results (RtHit, or one byte per ray
 * for any_hit) to h_out.  RT_ERR_CAPACITY if the request can never fit the
 * staging pool.  *ticket identifies it for rtServer_wait. */
int rtServer_submit(RtServer_t s, int scene, int any_hit, const RtRay* h_rays, int n, void* h_out,
                    uint64_t* ticket);
/* Device-buffer request (no staging, no footprint): rays and results stay in
 * the caller's device memory. */
int rtServer_submitDevice(RtServer_t s, int scene, int any_hit, const RtRay* d_rays, int n, void* d_out,
                          uint64_t* ticket);
/* Waits up to timeout_ms (< 0: no limit) for a request; RT_ERR_TIMEOUT if it
 * is not done (the ticket stays valid), else its status; info optional. */
int rtServer_wait(RtServer_t s, uint64_t ticket, int timeout_ms, RtRequestInfo* info);
int rtServer_getStats(RtServer_t s, RtServerStats* st);
/* Finishes every submitted request, then frees the server. */
void rtServer_destroy(RtServer_t s);

#ifdef __cplusplus
}
#endif

#endif /* RT_B200_H */
