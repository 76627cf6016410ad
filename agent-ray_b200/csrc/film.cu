// Film output on the device: Film::to_rgb_image (src/film.rs:276-302) with
// tonemap_pixel (:153-181).  One thread per pixel; every multiply and add is
// rounded separately in the reference's order (this file is compiled with
// -fmad=false), the divisions are IEEE, and powf is CUDA's (within 2 ulp of
// the host libm, so an 8-bit value can differ by one where the encoded value
// sits on a rounding boundary).
#include <algorithm>

#include "ar_internal.hpp"

namespace ar {

namespace {

__device__ __forceinline__ float luminance(float r, float g, float b) {
    return (0.2126f * r + 0.7152f * g) + 0.0722f * b;
}

__device__ __forceinline__ uint8_t to_u8(float e) {
    // (e * 255 + 0.5).min(255) as u8: Rust's cast truncates and saturates (NaN -> 0)
    const float v = fminf(e * 255.0f + 0.5f, 255.0f);
    return v > 0.0f ? uint8_t(v) : uint8_t(0);
}

__global__ void k_to_rgb8(const float* __restrict__ hdr, uint32_t n, uint32_t tm, float white_point, float inv_gamma,
                          float scale, uint8_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float c[3] = {hdr[3 * i] * scale, hdr[3 * i + 1] * scale, hdr[3 * i + 2] * scale};
        float s = 1.0f;
        if (tm == AR_TONEMAP_REINHARD) {
            const float lum = luminance(c[0], c[1], c[2]);
            s = lum > 1e-6f ? (lum / (1.0f + lum)) / lum : 1.0f / (1.0f + lum);
        } else if (tm == AR_TONEMAP_REINHARD_EXTENDED) {
            const float lw2 = white_point * white_point;
            const float lum = luminance(c[0], c[1], c[2]);
            const float mapped = (lum * (1.0f + lum / lw2)) / (1.0f + lum);
            s = lum > 1e-6f ? mapped / lum : 1.0f;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float m = tm == AR_TONEMAP_CLAMP ? c[k] : c[k] * s;
            m = fminf(fmaxf(m, 0.0f), 1.0f);
            out[3 * i + k] = to_u8(powf(m, inv_gamma));
        }
    }
}

}  // namespace

void film_to_rgb8(ar_context* ctx, const float* hdr, uint32_t w, uint32_t h, uint32_t tm, float white_point,
                  float gamma, float scale, uint8_t* out, bool on_device) {
    AR_REQUIRE(tm <= AR_TONEMAP_REINHARD_EXTENDED, AR_ERR_INVALID_ARGUMENT, "unknown tone mapper");
    AR_REQUIRE(gamma > 0.f, AR_ERR_INVALID_ARGUMENT, "gamma must be positive");
    AR_REQUIRE(tm != AR_TONEMAP_REINHARD_EXTENDED || white_point > 0.f, AR_ERR_INVALID_ARGUMENT,
               "white point must be positive");
    const size_t n = size_t(w) * h;
    AR_REQUIRE(n > 0 && n < (size_t(1) << 32), AR_ERR_INVALID_ARGUMENT, "bad image size");
    const float* src = hdr;
    uint8_t* dst = out;
    if (!on_device) {
        ctx->io.ensure(n * 3 * sizeof(float) + n * 3 + 256);
        float* d_hdr = ctx->io.buf.as<float>();
        dst = reinterpret_cast<uint8_t*>(d_hdr + 3 * n);
        AR_CUDA(cudaMemcpyAsync(d_hdr, hdr, n * 3 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        src = d_hdr;
    }
    const int grid = std::max(1, std::min(int((n + 255) / 256), ctx->num_sms * 8));
    k_to_rgb8<<<grid, 256, 0, ctx->stream>>>(src, uint32_t(n), tm, white_point, 1.0f / gamma, scale, dst);
    AR_CUDA(cudaGetLastError());
    if (!on_device) {
        AR_CUDA(cudaMemcpyAsync(out, dst, n * 3, cudaMemcpyDeviceToHost, ctx->stream));
        AR_CUDA(cudaStreamSynchronize(ctx->stream));
    }
}

}  // namespace ar

extern "C" int ar_film_to_rgb8(ar_context* ctx, const float* hdr_rgb, uint32_t width, uint32_t height,
                               uint32_t tone_mapper, float white_point, float gamma, float scale, uint8_t* out_rgb8,
                               uint32_t on_device) {
    return ar::guarded([&] {
        AR_REQUIRE(ctx && hdr_rgb && out_rgb8, AR_ERR_INVALID_ARGUMENT, "null argument");
        AR_CUDA(cudaSetDevice(ctx->device));
        ar::film_to_rgb8(ctx, hdr_rgb, width, height, tone_mapper, white_point, gamma, scale, out_rgb8,
                         on_device != 0);
    });
}
