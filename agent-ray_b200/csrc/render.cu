// ar_render dispatch: Integrator::render for PT, BDPT and GDPT
// (src/integrators/mod.rs:18-26), returning Film::to_hdr_vec-style output.
#include <cmath>

#include "ar_render.hpp"

namespace ar {

void check_device_flag(ar_context* ctx);

namespace {

struct V {
    float x, y, z;
};
inline V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V mul(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V divs(V a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dotv(V a, V b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V crossv(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V norm(V a) { return mul(a, 1.0f / std::sqrt(dotv(a, a))); }
inline void put(float* d, V v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; }

__global__ void k_film_to_f32(size_t n, const double* in, float* out) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = float(in[i]);
}

}  // namespace

CameraDev make_camera(const ar_camera_desc& d) {
    // PinholeCamera::from_lookat (src/cameras.rs:91-123), f32 throughout.
    V lf{d.lookfrom[0], d.lookfrom[1], d.lookfrom[2]};
    V la{d.lookat[0], d.lookat[1], d.lookat[2]};
    V up{d.vup[0], d.vup[1], d.vup[2]};
    const float rads_per_deg = 3.14159265358979323846f / 180.0f;
    const float theta = d.vfov_deg * rads_per_deg;
    const float hh = std::tan(theta / 2.0f);
    const float vh = 2.0f * hh;
    const float vw = d.aspect * vh;
    V w = norm(sub(lf, la));
    V u = norm(crossv(up, w));
    V v = crossv(w, u);
    V hor = mul(u, vw);
    V ver = mul(v, vh);
    V ll = sub(sub(sub(lf, divs(hor, 2.0f)), divs(ver, 2.0f)), w);
    CameraDev c{};
    put(c.o, lf);
    put(c.ll, ll);
    put(c.hor, hor);
    put(c.ver, ver);
    put(c.fwd, mul(w, -1.0f));
    c.area = vw * vh;
    put(c.right, norm(hor));
    put(c.up, norm(ver));
    c.vw = std::sqrt(dotv(hor, hor));
    c.vh = std::sqrt(dotv(ver, ver));
    return c;
}

void film_to_f32(ar_context* ctx, const void* film, bool f64, size_t count, float* out) {
    if (!f64) {
        AR_CUDA(cudaMemcpyAsync(out, film, count * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
        return;
    }
    const int grid = std::max(1, std::min(int((count + 255) / 256), ctx->num_sms * 8));
    k_film_to_f32<<<grid, 256, 0, ctx->stream>>>(count, static_cast<const double*>(film), out);
    AR_CUDA(cudaGetLastError());
}

void render(ar_context* ctx, const ar_scene* sc, const ar_camera_desc& camd, const ar_integrator_cfg& cfg,
            uint32_t w, uint32_t h, float* out, bool out_on_device) {
    AR_REQUIRE(cfg.integrator <= AR_INTEGRATOR_GDPT, AR_ERR_INVALID_ARGUMENT, "unknown integrator");
    AR_REQUIRE(cfg.film_precision <= AR_FILM_F64, AR_ERR_INVALID_ARGUMENT, "unknown film precision");
    AR_REQUIRE(uint64_t(w) * h <= (1ull << 28), AR_ERR_INVALID_ARGUMENT, "image too large");
    const CameraDev cam = make_camera(camd);
    const size_t count = size_t(w) * h * 3;
    const bool f64 = cfg.film_precision == AR_FILM_F64;
    const size_t film_bytes = count * (f64 ? sizeof(double) : sizeof(float));
    const int nfilms = cfg.integrator == AR_INTEGRATOR_GDPT ? 3 : 1;
    Workspace& films = ctx->films;
    films.ensure(film_bytes * nfilms + count * sizeof(float) * (nfilms + 1));
    float* dev_out_tmp = reinterpret_cast<float*>(films.buf.as<char>() + film_bytes * nfilms);
    float* dev_out = out_on_device ? out : dev_out_tmp;
    if (cfg.integrator == AR_INTEGRATOR_PT) {
        render_pt_films(ctx, sc, cam, cfg, w, h, false, films.buf.ptr);
        film_to_f32(ctx, films.buf.ptr, f64, count, dev_out);
    } else if (cfg.integrator == AR_INTEGRATOR_BDPT) {
        render_bdpt_film(ctx, sc, cam, cfg, w, h, films.buf.ptr);
        film_to_f32(ctx, films.buf.ptr, f64, count, dev_out);
    } else {
        render_pt_films(ctx, sc, cam, cfg, w, h, true, films.buf.ptr);
        float* f32films = dev_out_tmp + count;  // primal, dx, dy as f32
        for (int f = 0; f < 3; ++f)
            film_to_f32(ctx, films.buf.as<char>() + f * film_bytes, f64, count, f32films + f * count);
        poisson_reconstruct(ctx, cfg, w, h, f32films, f32films + count, f32films + 2 * count, dev_out, nullptr);
    }
    // Device output stays asynchronous on the context stream (errors surface at
    // the next ar_context_synchronize); host output synchronises here.
    if (!out_on_device) {
        AR_CUDA(cudaMemcpyAsync(out, dev_out, count * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        check_device_flag(ctx);
    }
}


}  // namespace ar
