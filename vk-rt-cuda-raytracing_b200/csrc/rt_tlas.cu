// rt_tlas.cu -- TLAS over instanced BLASes: GPU build and two-level
// closest/any-hit traversal (the two-level walk of layer/rt_ir_exec.cu:93-189
// and the instance records of layer/VkLayer_CudaRT.cpp:4517-4558, done on
// the compressed 8-wide layout).
//
// Build: world box of every instance = the 8 transformed corners of its
// BLAS root box, padded outward by a relative 2^-16 of the coordinate
// magnitudes (covers the rounding of the object-space ray transform), then
// the same GPU SAH builder with one instance per leaf.
// Trace: one stack for both levels.  Entering an instance transforms the
// world ray by the inverse 3x4 (no renormalisation, t stays in world units)
// and switches node/triangle arrays; node groups pushed at the top level
// carry a flag, so popping one restores the world ray.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "rt_internal.h"
#include "rt_trace.cuh"

namespace rtb {

constexpr uint32_t G_TOP = 1u << 16;   // group belongs to the top level
constexpr uint32_t G_INST = 1u << 17;  // group is a mask of instance leaves

template <bool ANY>
__global__ void __launch_bounds__(TRACE_T, TRACE_MINB)
    k_trace_tlas(const uint4* __restrict__ tnodes, const int* __restrict__ leaf_ids, const float4* __restrict__ inst,
                 const RtRay* __restrict__ rays, int n, RtHit* __restrict__ hits, int32_t* __restrict__ inst_out,
                 uint8_t* __restrict__ occ, int* __restrict__ work, int* __restrict__ status) {
    __shared__ uint2 sstack[SSTACK][TRACE_T];
    uint2 lstack[LSTACK];
    const int lane = threadIdx.x & 31;
    int ray = -1;
    bool exhausted = false;
    Ray wr, cr;
    Walk w;
    bool in_blas = false;
    const uint4* bnodes = nullptr;
    const float4* btris = nullptr;
    int cur_inst = -1;
    float thit = 0.f, hu = 0.f, hv = 0.f;
    int hprim = -1, hinst = -1;
    for (;;) {
        const bool need = ray < 0 && !exhausted;
        const unsigned want = __ballot_sync(FULL_MASK, need);
        if (want) {
            const int leader = __ffs(want) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(work, __popc(want));
            base = __shfl_sync(FULL_MASK, base, leader);
            if (need) {
                const int ri = base + __popc(want & ((1u << lane) - 1));
                if (ri < n) {
                    ray = ri;
                    wr = load_ray(rays, ri);
                    cr = wr;
                    in_blas = false;
                    thit = wr.tmax;
                    hprim = hinst = -1;
                    hu = hv = 0.f;
                    w.start();
                    w.ng = make_uint2(0u, (1u << wr.oct) | (1u << 8) | G_TOP);
                } else {
                    exhausted = true;
                }
            }
        }
        if (__all_sync(FULL_MASK, ray < 0)) break;
        if (ray < 0) continue;
        if (w.ng.y & G_INST) {
            // enter the next instance of an instance group
            uint32_t m = w.ng.y & 0xFFu;
            const int j = __ffs(m) - 1;
            m &= m - 1;
            const uint32_t base = w.ng.x;
            if (m) {
                if (!w.push(make_uint2(base, m | G_INST | G_TOP), sstack, lstack)) {
                    atomicOr(status, RT_STATUS_STACK);
                    hprim = -2;
                    goto finish;
                }
            }
            cur_inst = leaf_ids[base + j];
            const float4* ip = inst + (size_t)cur_inst * 4;
            const float4 r0 = __ldg(ip), r1 = __ldg(ip + 1), r2 = __ldg(ip + 2), pp = __ldg(ip + 3);
            const float m12[12] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w};
            float ox, oy, oz, dx, dy, dz;
            xform_point(m12, wr.ox, wr.oy, wr.oz, ox, oy, oz);
            xform_dir(m12, wr.dx, wr.dy, wr.dz, dx, dy, dz);
            cr = make_ray(make_float4(ox, oy, oz, wr.tmin), make_float4(dx, dy, dz, wr.tmax));
            bnodes = reinterpret_cast<const uint4*>(((unsigned long long)__float_as_uint(pp.y) << 32) | __float_as_uint(pp.x));
            btris = reinterpret_cast<const float4*>(((unsigned long long)__float_as_uint(pp.w) << 32) | __float_as_uint(pp.z));
            in_blas = true;
            w.ng = make_uint2(0u, (1u << cr.oct) | (1u << 8));
            continue;
        }
        {
            uint32_t tri_base = 0, tmask = 0;
            if (w.ng.y & 0xFFu) {
                uint32_t hitsm = w.ng.y & 0xFFu;
                const uint32_t imask = (w.ng.y >> 8) & 0xFFu;
                const uint32_t top = w.ng.y & G_TOP;
                const int k = __ffs(hitsm) - 1;
                hitsm &= hitsm - 1;
                const uint32_t slot = (uint32_t)k ^ cr.oct;
                const uint32_t ni = w.ng.x + __popc(imask & ((1u << slot) - 1));
                if (hitsm) {
                    if (!w.push(make_uint2(w.ng.x, hitsm | (imask << 8) | top), sstack, lstack)) {
                        atomicOr(status, RT_STATUS_STACK);
                        hprim = -2;
                        goto finish;
                    }
                }
                uint32_t nh;
                visit_node((top ? tnodes : bnodes) + (size_t)ni * 5, cr, thit, nh, tri_base, tmask, w.ng);
                if (top) {
                    w.ng.y |= G_TOP;
                    if (tmask) {
                        // instance leaves of this top node: keep the node group, walk the instances
                        if (w.ng.y & 0xFFu) {
                            if (!w.push(w.ng, sstack, lstack)) {
                                atomicOr(status, RT_STATUS_STACK);
                                hprim = -2;
                                goto finish;
                            }
                        }
                        w.ng = make_uint2(tri_base, (tmask & 0xFFu) | G_INST | G_TOP);
                        tmask = 0;
                        continue;
                    }
                }
            }
            while (tmask) {
                const int j = __ffs(tmask) - 1;
                tmask &= tmask - 1;
                const float4* tp = btris + (size_t)(tri_base + j) * 3;
                const float4 A = __ldg(tp), B = __ldg(tp + 1), Cc = __ldg(tp + 2);
                float t, u, v;
                if (intersect_tri(cr.ox, cr.oy, cr.oz, cr.dx, cr.dy, cr.dz, A, B, Cc, t, u, v)) {
                    const int prim = __float_as_int(A.w);
                    if (ANY) {
                        if (t > wr.tmin && t < wr.tmax) {
                            hprim = prim;
                            hinst = cur_inst;
                            goto finish;
                        }
                    } else if (t > wr.tmin &&
                               (t < thit || (t == thit && hprim >= 0 &&
                                             (cur_inst < hinst || (cur_inst == hinst && prim < hprim))))) {
                        thit = t;
                        hprim = prim;
                        hinst = cur_inst;
                        hu = u;
                        hv = v;
                    }
                }
            }
            if ((w.ng.y & 0xFFu) == 0) {
                if (w.sp == 0) goto finish;
                w.ng = w.pop(sstack, lstack);
                if (in_blas && (w.ng.y & G_TOP)) {
                    in_blas = false;
                    cr = wr;
                }
            }
        }
        continue;
    finish:
        if (ANY) {
            occ[ray] = hprim >= 0 ? 1 : 0;
        } else {
            reinterpret_cast<float4*>(hits)[ray] =
                make_float4(hprim >= 0 ? thit : __int_as_float(0x7f800000), __int_as_float(hprim >= 0 ? hprim : -1),
                            hprim >= 0 ? hu : 0.f, hprim >= 0 ? hv : 0.f);
            if (inst_out) inst_out[ray] = hprim >= 0 ? hinst : -1;
        }
        ray = -1;
    }
}

template <class K>
static int grid_for(K kernel) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, TRACE_T, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    return per_sm * num_sms();
}

int launch_trace_tlas(const CudaTLASHandle* t, const RtRay* rays, int n, RtHit* hits, int32_t* inst_out,
                      uint8_t* occ, int* work, int* status, cudaStream_t s) {
    const uint4* nodes = reinterpret_cast<const uint4*>(t->bvh8.nodes.p);
    if (occ) {
        static const int g = grid_for(k_trace_tlas<true>);
        k_trace_tlas<true><<<g, TRACE_T, 0, s>>>(nodes, t->bvh8.leaf_ids.p, t->inst.p, rays, n, hits, inst_out, occ,
                                                 work, status);
    } else {
        static const int g = grid_for(k_trace_tlas<false>);
        k_trace_tlas<false><<<g, TRACE_T, 0, s>>>(nodes, t->bvh8.leaf_ids.p, t->inst.p, rays, n, hits, inst_out,
                                                  occ, work, status);
    }
    return cudaGetLastError() == cudaSuccess ? RT_OK : RT_ERR_CUDA;
}

static float bits_f(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// inverse of a row-major affine 3x4 in double
static bool invert34(const float* m, double* inv) {
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
    const double A = e * i - f * h, B = -(d * i - f * g), Cc = d * h - e * g;
    const double det = a * A + b * B + c * Cc;
    if (!(fabs(det) > 1e-300)) return false;
    const double id = 1.0 / det;
    double r[9] = {A * id, -(b * i - c * h) * id, (b * f - c * e) * id,
                   B * id, (a * i - c * g) * id, -(a * f - c * d) * id,
                   Cc * id, -(a * h - b * g) * id, (a * e - b * d) * id};
    const double tx = m[3], ty = m[7], tz = m[11];
    for (int row = 0; row < 3; row++) {
        inv[row * 4 + 0] = r[row * 3 + 0];
        inv[row * 4 + 1] = r[row * 3 + 1];
        inv[row * 4 + 2] = r[row * 3 + 2];
        inv[row * 4 + 3] = -(r[row * 3 + 0] * tx + r[row * 3 + 1] * ty + r[row * 3 + 2] * tz);
    }
    return true;
}

}  // namespace rtb

using namespace rtb;

extern "C" {

CudaTLAS_t cudaTLAS_build(const CudaBVH_t* blas, int nb, const RtInstance* inst, int ni) {
    clear_error();
    if (!blas || nb <= 0 || !inst || ni <= 0) {
        set_error("cudaTLAS_build: empty input");
        return nullptr;
    }
    for (int i = 0; i < nb; i++)
        if (!blas[i]) {
            set_error("cudaTLAS_build: BLAS %d is NULL", i);
            return nullptr;
        }
    CudaTLASHandle* t = new (std::nothrow) CudaTLASHandle();
    if (!t) return nullptr;
    t->num_instances = ni;
    t->blas.assign(blas, blas + nb);
    t->h_inv.resize((size_t)ni * 12);
    std::vector<float4> rec((size_t)ni * 4), lo(ni), hi(ni);
    for (int k = 0; k < ni; k++) {
        const RtInstance& I = inst[k];
        if (I.blas < 0 || I.blas >= nb) {
            set_error("cudaTLAS_build: instance %d names BLAS %d of %d", k, I.blas, nb);
            delete t;
            return nullptr;
        }
        double inv[12];
        if (!invert34(I.xform, inv)) {
            set_error("cudaTLAS_build: instance %d transform is singular", k);
            delete t;
            return nullptr;
        }
        float* fi = &t->h_inv[(size_t)k * 12];
        for (int j = 0; j < 12; j++) fi[j] = (float)inv[j];
        const CudaBVHHandle* b = blas[I.blas];
        double wl[3] = {1e300, 1e300, 1e300}, wh[3] = {-1e300, -1e300, -1e300}, mag = 0.0;
        for (int c = 0; c < 8; c++) {
            const double p[3] = {(c & 1) ? b->bmax[0] : b->bmin[0], (c & 2) ? b->bmax[1] : b->bmin[1],
                                 (c & 4) ? b->bmax[2] : b->bmin[2]};
            for (int r = 0; r < 3; r++) {
                const double v = I.xform[r * 4] * p[0] + I.xform[r * 4 + 1] * p[1] + I.xform[r * 4 + 2] * p[2] +
                                 I.xform[r * 4 + 3];
                wl[r] = std::min(wl[r], v);
                wh[r] = std::max(wh[r], v);
                mag = std::max(mag, fabs(v));
            }
        }
        const double pad = ldexp(mag + (wh[0] - wl[0]) + (wh[1] - wl[1]) + (wh[2] - wl[2]), -16);
        lo[k] = make_float4(nextafterf((float)(wl[0] - pad), -INFINITY), nextafterf((float)(wl[1] - pad), -INFINITY),
                            nextafterf((float)(wl[2] - pad), -INFINITY), 0.f);
        hi[k] = make_float4(nextafterf((float)(wh[0] + pad), INFINITY), nextafterf((float)(wh[1] + pad), INFINITY),
                            nextafterf((float)(wh[2] + pad), INFINITY), 0.f);
        const unsigned long long np = (unsigned long long)b->bvh8.nodes.p, tp = (unsigned long long)b->bvh8.tris.p;
        rec[(size_t)k * 4 + 0] = make_float4(fi[0], fi[1], fi[2], fi[3]);
        rec[(size_t)k * 4 + 1] = make_float4(fi[4], fi[5], fi[6], fi[7]);
        rec[(size_t)k * 4 + 2] = make_float4(fi[8], fi[9], fi[10], fi[11]);
        rec[(size_t)k * 4 + 3] = make_float4(bits_f((uint32_t)np), bits_f((uint32_t)(np >> 32)), bits_f((uint32_t)tp),
                                             bits_f((uint32_t)(tp >> 32)));
    }
    DevBuf<float4> dlo, dhi;
    BuildConfig cfg;
    cfg.max_leaf = 1;
    bool ok = t->inst.alloc(rec.size()) && dlo.alloc(ni) && dhi.alloc(ni) &&
              RT_CUDA(cudaMemcpy(t->inst.p, rec.data(), rec.size() * sizeof(float4), cudaMemcpyHostToDevice)) &&
              RT_CUDA(cudaMemcpy(dlo.p, lo.data(), ni * sizeof(float4), cudaMemcpyHostToDevice)) &&
              RT_CUDA(cudaMemcpy(dhi.p, hi.data(), ni * sizeof(float4), cudaMemcpyHostToDevice)) &&
              build_bvh2(dlo.p, dhi.p, ni, cfg, t->bvh2, 0) && collapse_bvh8(t->bvh2, nullptr, t->bvh8, 0) &&
              ensure_counters(t->counters) && t->status.alloc(1) &&
              RT_CUDA(cudaMemset(t->status.p, 0, sizeof(int))) && RT_CUDA(cudaDeviceSynchronize()) &&
              (!getenv("RTB200_VALIDATE") || !atoi(getenv("RTB200_VALIDATE")) ||
               validate_bvh8(t->bvh8, t->bvh8.num_leaf_items, ni));
    if (!ok) {
        delete t;
        return nullptr;
    }
    return t;
}

void cudaTLAS_destroy(CudaTLAS_t t) {
    if (!t) return;
    cudaDeviceSynchronize();
    delete t;
}

int cudaTLAS_traceClosest(CudaTLAS_t t, const RtRay* d_rays, int n, RtHit* d_hits, int32_t* d_inst, void* stream) {
    if (!t || n < 0 || (n > 0 && (!d_rays || !d_hits))) {
        set_error("cudaTLAS_traceClosest: invalid argument");
        return RT_ERR_INVALID;
    }
    if (n == 0) return RT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    int* work = next_counter(t->counters, t->counter_next, s);
    const int rc = launch_trace_tlas(t, d_rays, n, d_hits, d_inst, nullptr, work, t->status.p, s);
    if (rc != RT_OK) RT_CUDA(cudaGetLastError());
    return rc;
}

int cudaTLAS_traceAny(CudaTLAS_t t, const RtRay* d_rays, int n, uint8_t* d_occ, void* stream) {
    if (!t || n < 0 || (n > 0 && (!d_rays || !d_occ))) {
        set_error("cudaTLAS_traceAny: invalid argument");
        return RT_ERR_INVALID;
    }
    if (n == 0) return RT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    int* work = next_counter(t->counters, t->counter_next, s);
    const int rc = launch_trace_tlas(t, d_rays, n, nullptr, nullptr, d_occ, work, t->status.p, s);
    if (rc != RT_OK) RT_CUDA(cudaGetLastError());
    return rc;
}

int cudaTLAS_getInverseTransforms(CudaTLAS_t t, float* out, int n) {
    if (!t || !out || n != t->num_instances) {
        set_error("cudaTLAS_getInverseTransforms: invalid argument");
        return RT_ERR_INVALID;
    }
    memcpy(out, t->h_inv.data(), t->h_inv.size() * sizeof(float));
    return RT_OK;
}

}  // extern "C"
