// Batched ray queries: closest hit (TLAS::intersect) and occlusion
// (Scene::occluded).  One thread per ray over SoA float4 ray records.
#include "ar_device.cuh"
#include "ar_internal.hpp"

namespace ar {

namespace {

template <bool kAnyHit>
__global__ void AR_TRAVERSAL_BOUNDS trace_kernel(DevScene sc, const float4* __restrict__ org_tmin,
                                                    const float4* __restrict__ dir_tmax, uint64_t n,
                                                    float4* __restrict__ hits, uint32_t* __restrict__ inst_ids,
                                                    uint8_t* __restrict__ occluded, int* err) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float4 a = __ldg(org_tmin + i), b = __ldg(dir_tmax + i);
        const Ray r = make_ray(mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w);
        HitRec h;
        traverse<kAnyHit>(sc, r, h, err);
        if (kAnyHit) {
            occluded[i] = h.slot != kInvalid ? 1 : 0;
        } else if (h.slot != kInvalid) {
            const uint32_t prim = __float_as_uint(__ldg(reinterpret_cast<const float*>(sc.tris + h.slot) + 3));
            hits[i] = make_float4(h.t, h.u, h.v, __uint_as_float(prim));
            inst_ids[i] = h.inst;
        } else {
            hits[i] = make_float4(INFINITY, 0.f, 0.f, __uint_as_float(kInvalid));
            inst_ids[i] = kInvalid;
        }
    }
}

}  // namespace

int trace_grid(const ar_context* ctx, uint64_t n) {
    const uint64_t blocks = (n + 127) / 128;
    const uint64_t cap = uint64_t(ctx->num_sms) * 16;
    return int(std::max<uint64_t>(1, std::min(blocks, cap)));
}

void launch_trace(ar_context* ctx, const ar_scene* sc, const float4* ot, const float4* dt, uint64_t n, bool any,
                  float4* hits, uint32_t* inst, uint8_t* occ) {
    if (n == 0) return;
    const int grid = trace_grid(ctx, n);
    KernelScope ks(ctx->prof, ctx->stream, any ? "trace_any" : "trace_closest");
    if (any)
        trace_kernel<true><<<grid, 128, 0, ctx->stream>>>(sc->view, ot, dt, n, nullptr, nullptr, occ,
                                                          ctx->err_flag.as<int>());
    else
        trace_kernel<false><<<grid, 128, 0, ctx->stream>>>(sc->view, ot, dt, n, hits, inst, nullptr,
                                                           ctx->err_flag.as<int>());
    AR_CUDA(cudaGetLastError());
}

}  // namespace ar
