// Integrator entry points behind ar_render (Integrator::render,
// src/integrators/mod.rs:18-26) and shared host-side helpers.
#pragma once
#include "ar_internal.hpp"

namespace ar {

// PinholeCamera (src/cameras.rs:91-248) in the layout the kernels read.
struct CameraDev {
    float o[3], ll[3], hor[3], ver[3], fwd[3];
    float area;
    float right[3], up[3];
    float vw, vh;
};

// PinholeCamera::from_lookat evaluated on the host in f32 (reference order).
CameraDev make_camera(const ar_camera_desc& d);

void render(ar_context* ctx, const ar_scene* sc, const ar_camera_desc& cam, const ar_integrator_cfg& cfg,
            uint32_t w, uint32_t h, float* out, bool out_on_device);

// Wavefront path tracer (PT, and GDPT base/offset paths).  Accumulates into
// device films (f32 or f64; GDPT: primal, dx, dy) already divided by spp.
void render_pt_films(ar_context* ctx, const ar_scene* sc, const CameraDev& cam, const ar_integrator_cfg& cfg,
                     uint32_t w, uint32_t h, bool gdpt, void* films);

// Bidirectional path tracer into a device film (f32 or f64) divided by spp.
void render_bdpt_film(ar_context* ctx, const ar_scene* sc, const CameraDev& cam, const ar_integrator_cfg& cfg,
                      uint32_t w, uint32_t h, void* film);

// Screened-Poisson reconstruction on the device.  Inputs are interleaved RGB
// f32 films (W*H*3); `out` receives the clamped reconstruction.
// Returns the number of kernels launched.
uint64_t poisson_reconstruct(ar_context* ctx, const ar_integrator_cfg& cfg, uint32_t w, uint32_t h, const float* primal,
                         const float* gx, const float* gy, float* out, double* rel_residual);

// Converts an f64 film to f32 (or copies an f32 film) into `out`.
void film_to_f32(ar_context* ctx, const void* film, bool f64, size_t count, float* out);

}  // namespace ar
