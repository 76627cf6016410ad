// Batched ray queries: closest hit (TLAS::intersect) and occlusion
// (Scene::occluded).  One thread per ray over SoA float4 ray records.
#include "ar_device.cuh"
#include "ar_internal.hpp"

namespace ar {

namespace {

template <bool kAnyHit>
__global__ void AR_TRAVERSAL_BOUNDS trace_kernel(const __grid_constant__ DevScene sc,
                                                    const float4* __restrict__ org_tmin,
                                                    const float4* __restrict__ dir_tmax, uint32_t n, uint32_t* cursor,
                                                    float4* __restrict__ hits, uint32_t* __restrict__ inst_ids,
                                                    uint8_t* __restrict__ occluded, int* err) {
    run_traversal<kAnyHit>(
        cursor, n, err,
        [&](uint32_t i, const DevScene*& s, Ray& r) {
            const float4 a = ld_once(org_tmin + i), b = ld_once(dir_tmax + i);
            s = &sc;
            r = make_ray(mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w);
        },
        [&](uint32_t i, const HitRec& h) {
            if (kAnyHit) {
                occluded[i] = h.slot != kInvalid ? 1 : 0;
            } else if (h.slot != kInvalid) {
                const uint32_t prim = __float_as_uint(__ldg(reinterpret_cast<const float*>(sc.tris + h.slot) + 3));
                st_once(hits + i, make_float4(h.t, h.u, h.v, __uint_as_float(prim)));
                st_once(inst_ids + i, h.inst);
            } else {
                st_once(hits + i, make_float4(INFINITY, 0.f, 0.f, __uint_as_float(kInvalid)));
                st_once(inst_ids + i, kInvalid);
            }
        });
}

}  // namespace

void launch_trace(ar_context* ctx, const ar_scene* sc, const float4* ot, const float4* dt, uint64_t n, bool any,
                  float4* hits, uint32_t* inst, uint8_t* occ) {
    if (n == 0) return;
    // Persistent grid; lanes fetch rays from a cursor.  Batches above 2^31 rays go in slices.
    const uint64_t kSlice = 1ull << 31;
    const int grid = std::max<int>(1, int(std::min<uint64_t>((n + 127) / 128,
                                                              uint64_t(ctx->num_sms) * ctx->trav_blocks_per_sm)));
    uint32_t* cursor = ctx->fetch.as<uint32_t>();
    KernelScope ks(ctx->prof, ctx->stream, any ? "trace_any" : "trace_closest");
    for (uint64_t off = 0; off < n; off += kSlice) {
        const uint32_t m = uint32_t(std::min(kSlice, n - off));
        AR_CUDA(cudaMemsetAsync(cursor, 0, sizeof(uint32_t), ctx->stream));
        if (any)
            trace_kernel<true><<<grid, 128, 0, ctx->stream>>>(sc->view, ot + off, dt + off, m, cursor, nullptr,
                                                              nullptr, occ + off, ctx->err_flag.as<int>());
        else
            trace_kernel<false><<<grid, 128, 0, ctx->stream>>>(sc->view, ot + off, dt + off, m, cursor,
                                                               hits + off, inst + off, nullptr,
                                                               ctx->err_flag.as<int>());
        AR_CUDA(cudaGetLastError());
    }
}

}  // namespace ar
