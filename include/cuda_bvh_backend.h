/* cuda_bvh_backend.h -- drop-in C-ABI of the B200 ray traversal engine.
 *
 * Same symbols, signatures, ownership rules and error conventions as the
 * reference project's layer/cuda_bvh_backend.h:1-147, so VkLayer_CudaRT and
 * the OptiX shim link against libcudabvh_b200.so unchanged.  Each entry point
 * names the reference declaration it replaces.  Behavioural differences (all
 * deliberate) are noted inline.
 *
 * Ownership: the handle owns every buffer until cudaBVH_destroy; getters
 * return borrowed host pointers that stay valid until destroy;
 * cudaBVH_buildTLASFast returns malloc'd arrays the caller free()s.
 * Errors: handle-returning calls return NULL, trace calls return 0 (their
 * result is MRays/s), int calls return 0 on success and -1 on failure.  The
 * reason of the last failure on the calling thread is rtGetLastError()
 * (rt_b200.h).  No entry point aborts the process.
 */
#ifndef CUDA_BVH_BACKEND_H
#define CUDA_BVH_BACKEND_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque handle to a built BVH (reference :12-13). */
typedef struct CudaBVHHandle* CudaBVH_t;

/* One triangle, 9 floats, 36 bytes (reference :15-18). */
typedef struct {
    float v0[3], v1[3], v2[3];
} CudaTri;

/* Reference :20-21.  Copies the host triangles to the GPU and builds the
 * acceleration structure there (binned SAH, 32 bins, <= 4 triangles per
 * leaf, collapsed to the compressed 8-wide layout).  NULL on empty input or
 * failure. */
CudaBVH_t cudaBVH_build(const CudaTri* tris, int numTris);

/* Reference :23-24.  NULL is a no-op. */
void cudaBVH_destroy(CudaBVH_t bvh);

/* Reference :26-31.  side x side camera rays from (camOx,camOy,camOz) looking
 * down +z with direction normalize(u, v, 1), u, v = (p + 0.5)/side*2 - 1.
 * Writes hit distances (1e30 on a miss) to outHitT (host, may be NULL).
 * Returns MRays/s of the traversal kernel, 0 on error. */
float cudaBVH_tracePrimary(CudaBVH_t bvh, int side,
                           float camOx, float camOy, float camOz,
                           float* outHitT);

/* Reference :33-40.  Host SoA rays (t > 0); writes hit distances in the
 * caller's ray order (1e30 on a miss).  Returns MRays/s, 0 on error. */
float cudaBVH_traceDiffuse(CudaBVH_t bvh, int numRays,
                           const float* rayOx, const float* rayOy, const float* rayOz,
                           const float* rayDx, const float* rayDy, const float* rayDz,
                           float* outHitT);

/* Reference :42-47.  Look-at camera toward the scene centre (fov 0.6),
 * face-normal shading, RGBA8 into caller host memory.  0 on success. */
int cudaBVH_traceToRGBA(CudaBVH_t bvh, int width, int height,
                        float camOx, float camOy, float camOz,
                        uint32_t* outRGBA_host);

/* Reference :49-56.  Same image into caller device memory; outFmt 0=RGBA8,
 * 1=BGRA8, 2=RGBA16F, 3=RGBA32F.  Asynchronous on the default stream.  0 on
 * success. */
int cudaBVH_traceToGPUPtr(CudaBVH_t bvh, int width, int height,
                          float camOx, float camOy, float camOz,
                          void* d_outRGBA, int outFmt);

/* Reference :58-64.  Fire-and-forget trace into device memory on the
 * background tracer thread; the first call waits for its frame. */
void cudaBVH_traceToGPUAsync(CudaBVH_t bvh, int width, int height,
                             float camOx, float camOy, float camOz,
                             void* d_outRGBA, int outFmt);

/* Reference :66-73.  Background tracer renders into a double-buffered host
 * image; each call copies the last finished frame (bufSize bytes) to
 * h_outRGBA and queues the next one.  The first call waits.  0 on success. */
int cudaBVH_traceToHostPtr(CudaBVH_t bvh, int width, int height,
                           float camOx, float camOy, float camOz,
                           void* h_outRGBA, int outFmt, uint64_t bufSize);

/* Reference :75-78.  Imports an opaque-fd external memory object and returns
 * a device pointer to its first `size` bytes (NULL on failure). */
void* cudaBVH_importBufferFd(int fd, uint64_t size);

/* Reference :80-81.  Scene bbox centre and diagonal length. */
void cudaBVH_getBounds(CudaBVH_t bvh, float* centerX, float* centerY, float* centerZ, float* extent);

/* Reference :83-86.  Triangle count, BVH4 export node count, and the number
 * of compressed 8-wide nodes the traversal kernels use (the reference
 * returned its BVH4 count here). */
int cudaBVH_getNumTris(CudaBVH_t bvh);
int cudaBVH_getNumBVH4Nodes(CudaBVH_t bvh);
int cudaBVH_getNumCWBVHNodes(CudaBVH_t bvh);

/* Reference :88-91.  BVH4 export, 64 bytes per node: x, y, z bounds as 8
 * halfs each (4 mins then 4 maxs), then int child[4] (-1 empty, <= -2 leaf
 * -(start<<3 | count-1) - 2).  Bounds are rounded outward (the reference
 * rounded to nearest, which can shrink boxes). */
const void* cudaBVH_getNodeData(CudaBVH_t bvh);

/* Reference :93-96.  Nine host float arrays (v0x..v2z) in BVH leaf order. */
void cudaBVH_getTriData(CudaBVH_t bvh, const float* outPtrs[9]);

/* Reference :98-103.  Stackless BVH2, 8 u32 per node: bmin, bmax (fp32),
 * leaf_enc (0 inner, -(start<<3 | count-1) - 2 leaf), skip (next node after
 * the subtree, -1 at the end).  Returns the node count. */
int cudaBVH_getStacklessBVH2(CudaBVH_t bvh, uint32_t** outData);

/* Reference :105-111.  3 vec4 per triangle in leaf order:
 * {v0.xyz, v1.x}, {v1.yz, v2.xy}, {v2.z, original index as float, 0, 0}.
 * Returns the vec4 count. */
int cudaBVH_getPackedTris(CudaBVH_t bvh, float** outData);

/* Reference :113-116.  Synchronises and resets this process's CUDA context;
 * no CUDA call may follow. */
void cudaBVH_resetDevice(void);

/* Reference :118-123.  BVH over AABBs (6 floats each); leaf primitive index
 * = AABB index.  NULL on empty input. */
CudaBVH_t cudaBVH_buildFromAABBs(const float* aabbs, int numAABBs);

/* Reference :125-131.  Morton LBVH over AABBs (single-instance leaves) as a
 * stackless export; *outNodes (8 u32 per node) and *outOrdered (sorted
 * position -> AABB index) are malloc'd, caller frees.  Returns the node
 * count (0 on bad input).  Node bytes equal the reference's except that
 * every skip pointer is correct (the reference leaves -2 placeholders). */
#ifdef __cplusplus
int cudaBVH_buildTLASFast(const float* aabbs, int numAABBs, uint32_t** outNodes,
                          int** outOrdered = nullptr);
#else
int cudaBVH_buildTLASFast(const float* aabbs, int numAABBs, uint32_t** outNodes,
                          int** outOrdered);
#endif

/* Reference :133-141.  Copies `size` bytes at `offset` of an opaque-fd
 * external memory object to host memory.  0 on success, -1 on failure. */
int cudaBVH_readGPUMemoryFd(int fd, uint64_t allocationSize,
                            uint64_t offset, uint64_t size, void* dst);

#ifdef __cplusplus
}
#endif

#endif /* CUDA_BVH_BACKEND_H */
