// Film output on the device: Film::to_rgb_image (src/film.rs:276-302) with
// tonemap_pixel (:153-181).  One thread per pixel; every multiply and add is
// rounded separately in the reference's order (this file is compiled with
// -fmad=false), the divisions are IEEE, and powf is CUDA's (within 2 ulp of
// the host libm, so an 8-bit value can differ by one where the encoded value
// sits on a rounding boundary).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include <cuda_fp16.h>
#include <zlib.h>

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

// Film::save_exr (src/film.rs:304-346): linear RGB * scale as HALF channels in
// an OpenEXR scanline file with ZIP compression (16 scanlines per chunk).  A
// chunk's uncompressed bytes are, scanline by scanline, the B, G, then R
// channel (channels sorted by name), each `width` little-endian halves.  ZIP
// first moves the even-offset bytes before the odd-offset ones, then replaces
// every byte but the first by (byte - previous byte + 128) mod 256; only the
// deflate step that follows runs on the host.  Every value offset is even, so
// the first half of a reordered chunk is the low bytes of its halves in order
// and the second half their high bytes: thread g converts value g (and its
// predecessor) and writes both of its predicted bytes.
constexpr uint32_t kExrLinesPerChunk = 16;

__device__ __forceinline__ uint16_t exr_half(const float* rgb, uint32_t w, size_t v, float scale) {
    // value v of the file's channel order: row, then channel B/G/R, then x
    const size_t row = v / (3 * size_t(w));
    const uint32_t rem = uint32_t(v - row * 3 * w);
    const uint32_t c = 2 - rem / w, x = rem % w;
    const float a = rgb[(row * w + x) * 3 + c];
    const float f = a * scale;
    if (isnan(f)) {
        // The host's product keeps a NaN operand's sign and payload (SSE takes
        // the first NaN operand, quieted; an invalid product gives the default
        // NaN 0xffc00000), where the GPU's multiply returns one canonical NaN.
        // f16 conversion then keeps the sign and the top mantissa bits.
        const uint32_t b = isnan(a) ? (__float_as_uint(a) | 0x400000u)
                                    : isnan(scale) ? (__float_as_uint(scale) | 0x400000u) : 0xffc00000u;
        return uint16_t(((b >> 16) & 0x8000u) | 0x7e00u | ((b & 0x7fffffu) >> 13));
    }
    return __half_as_ushort(__float2half_rn(f));  // f16::from_f32: IEEE round to nearest even
}

__global__ void k_exr_pack(const float* __restrict__ rgb, uint32_t w, uint32_t h, float scale,
                           uint8_t* __restrict__ out) {
    const size_t n = size_t(w) * h * 3;
    const size_t per_chunk = size_t(kExrLinesPerChunk) * 3 * w;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const size_t start = (g / per_chunk) * per_chunk;  // first value of this chunk
        const size_t m = std::min(per_chunk, n - start);     // values in this chunk
        const size_t j = g - start;
        const uint16_t cur = exr_half(rgb, w, g, scale);
        uint8_t lo, hi;
        if (j == 0) {
            lo = uint8_t(cur & 0xff);
            const uint16_t last = exr_half(rgb, w, start + m - 1, scale);  // the byte before the high half
            hi = uint8_t(((cur >> 8) - (last & 0xff) + 384) & 0xff);
        } else {
            const uint16_t prev = exr_half(rgb, w, g - 1, scale);
            lo = uint8_t(((cur & 0xff) - (prev & 0xff) + 384) & 0xff);
            hi = uint8_t(((cur >> 8) - (prev >> 8) + 384) & 0xff);
        }
        out[2 * start + j] = lo;
        out[2 * start + m + j] = hi;
    }
}

// Undoes the predictor and the reorder of one chunk (for a chunk that deflate
// does not shrink, which the file then stores uncompressed).
void exr_unpack_chunk(const uint8_t* packed, size_t nbytes, uint8_t* raw) {
    std::vector<uint8_t> t(packed, packed + nbytes);
    for (size_t i = 1; i < nbytes; ++i) t[i] = uint8_t(t[i - 1] + t[i] - 128);
    const size_t half = (nbytes + 1) / 2;
    for (size_t i = 0; i < nbytes; ++i) raw[i] = (i & 1) ? t[half + i / 2] : t[i / 2];
}

void put_attr(std::vector<uint8_t>& f, const char* name, const char* type, const void* v, uint32_t size) {
    f.insert(f.end(), name, name + strlen(name) + 1);
    f.insert(f.end(), type, type + strlen(type) + 1);
    const uint8_t* sz = reinterpret_cast<const uint8_t*>(&size);
    f.insert(f.end(), sz, sz + 4);
    const uint8_t* b = static_cast<const uint8_t*>(v);
    f.insert(f.end(), b, b + size);
}

template <class T>
void put(std::vector<uint8_t>& f, T v) {
    const uint8_t* b = reinterpret_cast<const uint8_t*>(&v);
    f.insert(f.end(), b, b + sizeof(T));
}

}  // namespace

void film_save_exr(ar_context* ctx, const float* rgb, uint32_t w, uint32_t h, float scale, bool on_device,
                   const char* path) {
    const size_t npix = size_t(w) * h;
    AR_REQUIRE(w > 0 && h > 0 && npix < (size_t(1) << 31) / 3, AR_ERR_INVALID_ARGUMENT, "bad image size");
    const size_t nbytes = npix * 3 * 2;
    const float* src = rgb;
    ctx->io.ensure((on_device ? 0 : npix * 3 * sizeof(float)) + nbytes + 256);
    uint8_t* d_out = ctx->io.buf.as<uint8_t>();
    if (!on_device) {
        float* d_rgb = ctx->io.buf.as<float>();
        d_out = reinterpret_cast<uint8_t*>(d_rgb + 3 * npix);
        AR_CUDA(cudaMemcpyAsync(d_rgb, rgb, npix * 3 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        src = d_rgb;
    }
    const int grid = std::max(1, std::min(int((npix * 3 + 255) / 256), ctx->num_sms * 8));
    k_exr_pack<<<grid, 256, 0, ctx->stream>>>(src, w, h, scale, d_out);
    AR_CUDA(cudaGetLastError());
    std::vector<uint8_t> packed(nbytes);
    AR_CUDA(cudaMemcpyAsync(packed.data(), d_out, nbytes, cudaMemcpyDeviceToHost, ctx->stream));
    AR_CUDA(cudaStreamSynchronize(ctx->stream));

    // deflate the chunks on the host threads
    const uint32_t nchunks = (h + kExrLinesPerChunk - 1) / kExrLinesPerChunk;
    const size_t chunk_bytes = size_t(kExrLinesPerChunk) * w * 6;
    std::vector<std::vector<uint8_t>> data(nchunks);
    std::vector<int> zerr(nchunks, Z_OK);
    auto work = [&](uint32_t t, uint32_t nt) {
        for (uint32_t c = t; c < nchunks; c += nt) {
            const size_t off = size_t(c) * chunk_bytes, n = std::min(chunk_bytes, nbytes - off);
            uLongf zn = compressBound(uLong(n));
            data[c].resize(zn);
            zerr[c] = compress2(data[c].data(), &zn, packed.data() + off, uLong(n), Z_DEFAULT_COMPRESSION);
            if (zerr[c] == Z_OK && zn < n) {
                data[c].resize(zn);
            } else {  // stored raw: the plain scanline bytes
                data[c].resize(n);
                exr_unpack_chunk(packed.data() + off, n, data[c].data());
                zerr[c] = Z_OK;
            }
        }
    };
    const uint32_t nt = std::max(1u, std::min(nchunks, std::min(32u, std::thread::hardware_concurrency())));
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nt; ++t) pool.emplace_back(work, t, nt);
    work(0, nt);
    for (auto& th : pool) th.join();

    // header (attributes in name order), offset table, chunks
    std::vector<uint8_t> f;
    put<uint32_t>(f, 20000630u);  // magic
    put<uint32_t>(f, 2u);         // version 2, single-part scanline
    std::vector<uint8_t> ch;
    for (const char* name : {"B", "G", "R"}) {
        ch.push_back(uint8_t(name[0]));
        ch.push_back(0);
        put<int32_t>(ch, 1);  // HALF
        put<uint32_t>(ch, 0); // pLinear + reserved
        put<int32_t>(ch, 1);  // x sampling
        put<int32_t>(ch, 1);  // y sampling
    }
    ch.push_back(0);
    put_attr(f, "channels", "chlist", ch.data(), uint32_t(ch.size()));
    const uint8_t zip = 3;  // ZIP_COMPRESSION: 16 scanlines per chunk
    put_attr(f, "compression", "compression", &zip, 1);
    const int32_t box[4] = {0, 0, int32_t(w) - 1, int32_t(h) - 1};
    put_attr(f, "dataWindow", "box2i", box, 16);
    put_attr(f, "displayWindow", "box2i", box, 16);
    const uint8_t increasing_y = 0;
    put_attr(f, "lineOrder", "lineOrder", &increasing_y, 1);
    put_attr(f, "name", "string", "beauty", 6);  // LayerAttributes::named("beauty")
    const float one = 1.0f, centre[2] = {0.f, 0.f};
    put_attr(f, "pixelAspectRatio", "float", &one, 4);
    put_attr(f, "screenWindowCenter", "v2f", centre, 8);
    put_attr(f, "screenWindowWidth", "float", &one, 4);
    f.push_back(0);  // end of header
    uint64_t at = f.size() + 8 * uint64_t(nchunks);
    for (uint32_t c = 0; c < nchunks; ++c) {
        put<uint64_t>(f, at);
        at += 8 + data[c].size();
    }
    for (uint32_t c = 0; c < nchunks; ++c) {
        put<int32_t>(f, int32_t(c * kExrLinesPerChunk));
        put<int32_t>(f, int32_t(data[c].size()));
        f.insert(f.end(), data[c].begin(), data[c].end());
    }
    FILE* fp = std::fopen(path, "wb");
    AR_REQUIRE(fp, AR_ERR_INVALID_ARGUMENT, "cannot open the output file");
    const size_t wrote = std::fwrite(f.data(), 1, f.size(), fp);
    const int closed = std::fclose(fp);
    AR_REQUIRE(wrote == f.size() && closed == 0, AR_ERR_INTERNAL, "writing the EXR file failed");
}

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

extern "C" int ar_film_save_exr(ar_context* ctx, const float* hdr_rgb, uint32_t width, uint32_t height, float scale,
                                uint32_t on_device, const char* path) {
    return ar::guarded([&] {
        AR_REQUIRE(ctx && hdr_rgb && path, AR_ERR_INVALID_ARGUMENT, "null argument");
        AR_CUDA(cudaSetDevice(ctx->device));
        ar::film_save_exr(ctx, hdr_rgb, width, height, scale, on_device != 0, path);
    });
}
