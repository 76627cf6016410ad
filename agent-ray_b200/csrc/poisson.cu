// Screened-Poisson reconstruction for the gradient-domain tracer
// (screened_poisson_reconstruct, src/integrators/gradient_domain_pt.rs:449-630).
//
// System per colour channel (5-point stencil, Neumann borders):
//   (alpha + N(x)) I(x) - sum_{n in N(x)} I(n) = alpha * primal(x) + div G(x)
// (the reference's sign; AR_GDPT_CONSISTENT_DIVERGENCE subtracts div G instead)
//
// Two solvers:
//   * red-black SOR, the reference method: each half sweep updates one colour
//     of the checkerboard, whose neighbours all have the other colour, so the
//     sweep is order independent and matches the sequential loop bit for bit
//     (this file is compiled with -fmad=false);
//   * FP32 conjugate gradient with FP64 iterative refinement: the residual
//     r = b - A x and all dot products are accumulated in FP64, the correction
//     A d = r is solved in FP32 CG, and x (FP64) += d until ||r|| / ||b|| <= tol.
// Buffers are interleaved RGB (W*H*3), like Film::to_hdr_vec.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ar_render.hpp"

namespace ar {

namespace {

__global__ void k_rhs(uint32_t w, uint32_t h, const float* __restrict__ primal, const float* __restrict__ gx,
                      const float* __restrict__ gy, float alpha, bool neg_div, float* __restrict__ rhs,
                      float* __restrict__ img) {
    const uint32_t n = w * h;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t x = i % w, y = i / w;
        for (int c = 0; c < 3; ++c) {
            float div = gx[3 * i + c];
            if (x > 0) div -= gx[3 * (i - 1) + c];
            div += gy[3 * i + c];
            if (y > 0) div -= gy[3 * (i - w) + c];
            const float a = alpha * primal[3 * i + c];
            rhs[3 * i + c] = neg_div ? a - div : a + div;
            img[3 * i + c] = primal[3 * i + c];
        }
    }
}

// One red-black half sweep over pixels with (x + y) & 1 == parity.
__global__ void k_sor_half(uint32_t w, uint32_t h, uint32_t parity, const float* __restrict__ rhs, float* img,
                           float alpha, float omega) {
    const uint32_t half_w = (w + 1) / 2;
    const uint32_t n = half_w * h;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t y = k / half_w;
        const uint32_t x = 2 * (k - y * half_w) + ((y + parity) & 1u);
        if (x >= w) continue;
        const uint32_t i = y * w + x;
        uint32_t nn = 0;
        float s0 = 0.f, s1 = 0.f, s2 = 0.f;
        if (x > 0) { s0 += img[3 * (i - 1)]; s1 += img[3 * (i - 1) + 1]; s2 += img[3 * (i - 1) + 2]; nn++; }
        if (x + 1 < w) { s0 += img[3 * (i + 1)]; s1 += img[3 * (i + 1) + 1]; s2 += img[3 * (i + 1) + 2]; nn++; }
        if (y > 0) { s0 += img[3 * (i - w)]; s1 += img[3 * (i - w) + 1]; s2 += img[3 * (i - w) + 2]; nn++; }
        if (y + 1 < h) { s0 += img[3 * (i + w)]; s1 += img[3 * (i + w) + 1]; s2 += img[3 * (i + w) + 2]; nn++; }
        const float diag = alpha + float(nn);
        const float inv = 1.0f / diag;
        const float g0 = (rhs[3 * i] + s0) * inv, g1 = (rhs[3 * i + 1] + s1) * inv, g2 = (rhs[3 * i + 2] + s2) * inv;
        img[3 * i] = (1.0f - omega) * img[3 * i] + omega * g0;
        img[3 * i + 1] = (1.0f - omega) * img[3 * i + 1] + omega * g1;
        img[3 * i + 2] = (1.0f - omega) * img[3 * i + 2] + omega * g2;
    }
}

__global__ void k_clamp(size_t n, const float* __restrict__ in, float* __restrict__ out) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = in[i] > 0.f ? in[i] : 0.f;
}

// ---- CG ----
template <class T>
__device__ __forceinline__ void stencil(uint32_t w, uint32_t h, uint32_t i, const T* v, double alpha, double out[3]) {
    const uint32_t x = i % w, y = i / w;
    double s[3] = {0, 0, 0};
    int nn = 0;
    auto add = [&](uint32_t j) { for (int c = 0; c < 3; ++c) s[c] += double(v[3 * j + c]); nn++; };
    if (x > 0) add(i - 1);
    if (x + 1 < w) add(i + 1);
    if (y > 0) add(i - w);
    if (y + 1 < h) add(i + w);
    for (int c = 0; c < 3; ++c) out[c] = (alpha + nn) * double(v[3 * i + c]) - s[c];
}

__device__ __forceinline__ void block_add3(double a0, double a1, double a2, double* dst) {
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_down_sync(0xffffffffu, a0, o);
        a1 += __shfl_down_sync(0xffffffffu, a1, o);
        a2 += __shfl_down_sync(0xffffffffu, a2, o);
    }
    __shared__ double sm[3][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sm[0][wid] = a0; sm[1][wid] = a1; sm[2][wid] = a2; }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        a0 = lane < nw ? sm[0][lane] : 0.0;
        a1 = lane < nw ? sm[1][lane] : 0.0;
        a2 = lane < nw ? sm[2][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_down_sync(0xffffffffu, a0, o);
            a1 += __shfl_down_sync(0xffffffffu, a1, o);
            a2 += __shfl_down_sync(0xffffffffu, a2, o);
        }
        if (lane == 0) { atomicAdd(dst, a0); atomicAdd(dst + 1, a1); atomicAdd(dst + 2, a2); }
    }
    __syncthreads();
}

// b (f64) = alpha*primal + div G; x (f64) = primal; bb += |b|^2.
__global__ void k_cg_setup(uint32_t w, uint32_t h, const float* primal, const float* gx, const float* gy, double alpha,
                           bool neg_div, double* b, double* x, double* bb) {
    const uint32_t n = w * h;
    double a[3] = {0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t xx = i % w, yy = i / w;
        for (int c = 0; c < 3; ++c) {
            double div = gx[3 * i + c];
            if (xx > 0) div -= gx[3 * (i - 1) + c];
            div += gy[3 * i + c];
            if (yy > 0) div -= gy[3 * (i - w) + c];
            const double av = alpha * double(primal[3 * i + c]);
            const double bv = neg_div ? av - div : av + div;
            b[3 * i + c] = bv;
            x[3 * i + c] = primal[3 * i + c];
            a[c] += bv * bv;
        }
    }
    block_add3(a[0], a[1], a[2], bb);
}

// r (f32) = b - A x (f64 arithmetic); p = r; d = 0; rr += |r|^2 (f64).
__global__ void k_cg_residual(uint32_t w, uint32_t h, const double* b, const double* x, double alpha, float* r,
                              float* p, float* d, double* rr) {
    const uint32_t n = w * h;
    double a[3] = {0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ax[3];
        stencil(w, h, i, x, alpha, ax);
        for (int c = 0; c < 3; ++c) {
            const double rv = b[3 * i + c] - ax[c];
            r[3 * i + c] = float(rv);
            p[3 * i + c] = float(rv);
            d[3 * i + c] = 0.f;
            a[c] += rv * rv;
        }
    }
    block_add3(a[0], a[1], a[2], rr);
}

// q = A p (f32 storage, f64 accumulation); pq += p.q
__global__ void k_cg_matvec(uint32_t w, uint32_t h, const float* p, double alpha, float* q, double* pq) {
    const uint32_t n = w * h;
    double a[3] = {0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ap[3];
        stencil(w, h, i, p, alpha, ap);
        for (int c = 0; c < 3; ++c) {
            q[3 * i + c] = float(ap[c]);
            a[c] += double(p[3 * i + c]) * ap[c];
        }
    }
    block_add3(a[0], a[1], a[2], pq);
}

// scal layout (f64): [0..3) rr, [3..6) pq, [6..9) rr_new
__global__ void k_cg_update(uint32_t n, const float* p, const float* q, float* d, float* r, const double* scal,
                            double* rr_new) {
    float al[3];
    for (int c = 0; c < 3; ++c) al[c] = scal[3 + c] != 0.0 ? float(scal[c] / scal[3 + c]) : 0.f;
    double a[3] = {0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int c = 0; c < 3; ++c) {
            d[3 * i + c] += al[c] * p[3 * i + c];
            const float rv = r[3 * i + c] - al[c] * q[3 * i + c];
            r[3 * i + c] = rv;
            a[c] += double(rv) * double(rv);
        }
    }
    block_add3(a[0], a[1], a[2], rr_new);
}

__global__ void k_cg_direction(uint32_t n, const float* r, float* p, const double* scal) {
    float be[3];
    for (int c = 0; c < 3; ++c) be[c] = scal[c] != 0.0 ? float(scal[6 + c] / scal[c]) : 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c) p[3 * i + c] = r[3 * i + c] + be[c] * p[3 * i + c];
}

// rr <- rr_new; pq, rr_new <- 0
__global__ void k_cg_rotate(double* scal) {
    if (threadIdx.x < 3) {
        scal[threadIdx.x] = scal[6 + threadIdx.x];
        scal[3 + threadIdx.x] = 0.0;
        scal[6 + threadIdx.x] = 0.0;
    }
}

__global__ void k_cg_accumulate(size_t n, double* x, const float* d) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        x[i] += double(d[i]);
}

__global__ void k_cg_output(size_t n, const double* x, float* out) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = x[i] > 0.0 ? float(x[i]) : 0.f;
}

}  // namespace

// The red-black SOR solve with caller-provided scratch (rhs and img, 3*W*H
// floats each) on `stream`; launches only, no allocation, no synchronisation.
void poisson_sor_with_scratch(cudaStream_t stream, int num_sms, const ar_integrator_cfg& cfg, uint32_t w, uint32_t h,
                              const float* primal, const float* gx, const float* gy, float* rhs, float* img,
                              float* out) {
    const size_t n = size_t(w) * h;
    const int grid = std::max(1, std::min(int((n + 255) / 256), num_sms * 8));
    k_rhs<<<grid, 256, 0, stream>>>(w, h, primal, gx, gy, cfg.alpha,
                                     (cfg.gdpt_flags & AR_GDPT_CONSISTENT_DIVERGENCE) != 0, rhs, img);
    for (uint32_t it = 0; it < cfg.poisson_iterations; ++it)
        for (uint32_t parity = 0; parity < 2; ++parity)
            k_sor_half<<<grid, 256, 0, stream>>>(w, h, parity, rhs, img, cfg.alpha, cfg.sor_omega);
    k_clamp<<<grid, 256, 0, stream>>>(3 * n, img, out);
    AR_CUDA(cudaGetLastError());
}

uint64_t poisson_reconstruct(ar_context* ctx, const ar_integrator_cfg& cfg, uint32_t w, uint32_t h, const float* primal,
                         const float* gx, const float* gy, float* out, double* rel_residual) {
    const size_t n = size_t(w) * h;
    const int grid = std::max(1, std::min(int((n + 255) / 256), ctx->num_sms * 8));
    cudaStream_t st = ctx->stream;
    if (cfg.poisson_solver == AR_POISSON_SOR) {
        ctx->solver.ensure(2 * 3 * n * sizeof(float));
        float* rhs = ctx->solver.buf.as<float>();
        poisson_sor_with_scratch(st, ctx->num_sms, cfg, w, h, primal, gx, gy, rhs, rhs + 3 * n, out);
        if (rel_residual) *rel_residual = -1.0;
        return 2 + 2 * uint64_t(cfg.poisson_iterations);
    }
    // CG with FP64 refinement.
    const double alpha = double(cfg.alpha);
    const double tol = cfg.poisson_tolerance > 0 ? cfg.poisson_tolerance : 1e-6;
    const uint32_t max_total = cfg.poisson_iterations ? cfg.poisson_iterations : 1000;
    const uint32_t inner = 32;
    ctx->solver.ensure(3 * n * (2 * sizeof(double) + 4 * sizeof(float)) + 16 * sizeof(double) + 1024);
    double* b = ctx->solver.buf.as<double>();
    double* x = b + 3 * n;
    float* r = reinterpret_cast<float*>(x + 3 * n);
    float* p = r + 3 * n;
    float* q = p + 3 * n;
    float* d = q + 3 * n;
    double* scal = reinterpret_cast<double*>(d + 3 * n + 64);
    scal = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(scal) + 63) & ~uintptr_t(63));
    double* bb = scal + 9;
    AR_CUDA(cudaMemsetAsync(scal, 0, 16 * sizeof(double), st));
    k_cg_setup<<<grid, 256, 0, st>>>(w, h, primal, gx, gy, alpha,
                                     (cfg.gdpt_flags & AR_GDPT_CONSISTENT_DIVERGENCE) != 0, b, x, bb);
    double hb[16];
    double res = 0.0;
    uint32_t total = 0;
    uint64_t launches = 1;
    for (;;) {
        AR_CUDA(cudaMemsetAsync(scal, 0, 9 * sizeof(double), st));
        k_cg_residual<<<grid, 256, 0, st>>>(w, h, b, x, alpha, r, p, d, scal);
        launches++;
        AR_CUDA(cudaMemcpyAsync(hb, scal, 12 * sizeof(double), cudaMemcpyDeviceToHost, st));
        AR_CUDA(cudaStreamSynchronize(st));
        res = 0.0;
        for (int c = 0; c < 3; ++c) {
            const double bn = hb[9 + c] > 0 ? std::sqrt(hb[9 + c]) : 1.0;
            res = std::max(res, std::sqrt(hb[c]) / bn);
        }
        if (res <= tol || total >= max_total) break;
        for (uint32_t k = 0; k < inner; ++k) {
            k_cg_matvec<<<grid, 256, 0, st>>>(w, h, p, alpha, q, scal + 3);
            k_cg_update<<<grid, 256, 0, st>>>(uint32_t(n), p, q, d, r, scal, scal + 6);
            k_cg_direction<<<grid, 256, 0, st>>>(uint32_t(n), r, p, scal);
            k_cg_rotate<<<1, 32, 0, st>>>(scal);
        }
        total += inner;
        k_cg_accumulate<<<grid, 256, 0, st>>>(3 * n, x, d);
        launches += 4 * inner + 1;
    }
    k_cg_output<<<grid, 256, 0, st>>>(3 * n, x, out);
    AR_CUDA(cudaGetLastError());
    AR_CUDA(cudaStreamSynchronize(st));
    if (rel_residual) *rel_residual = res;
    return launches + 1;
}

}  // namespace ar
