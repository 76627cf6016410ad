// ar_poisson_sor_static: the screened-Poisson red-black SOR solve for callers
// that cannot allocate device memory.
//
// Some hosts of this library must not call cudaMalloc/cudaFree while they
// render: a real-time frame loop or a plugin inside another application whose
// memory manager owns the whole device pool (and treats any foreign
// allocation as a budget violation), or code that runs between CUDA-graph
// captures where an allocation would implicitly synchronise the device.  This
// entry point takes device pointers for its inputs and output, creates no
// context, and keeps its scratch (the right-hand side and the iterate, 3*W*H
// floats each) in a file-scope device array that every GPU loading the library
// holds until the process exits.
//
// The array's name, used from host code, is only a host-side stand-in: its
// device address is looked up once per device with cudaGetSymbolAddress (the
// first call on each device does that set-up, with that device current, and
// should therefore come before any stream capture).  All calls share the one
// array, so calls that overlap on the GPU (different streams, or different
// host threads on one device) race on it and must be serialised by the
// caller; a later call overwrites every element it reads, so no state carries
// over from the previous call.
#include <mutex>
#include <string>

#include "ar_render.hpp"

namespace ar {

void poisson_sor_with_scratch(cudaStream_t stream, int num_sms, const ar_integrator_cfg& cfg, uint32_t w, uint32_t h,
                              const float* primal, const float* gx, const float* gy, float* rhs, float* img,
                              float* out);

namespace {

constexpr uint32_t kStaticSorMaxPixels = AR_STATIC_SOR_MAX_PIXELS;

// rhs followed by img, each 3 * kStaticSorMaxPixels floats (6 MiB in total).
static __device__ __align__(256) float g_sor_scratch[2 * 3 * size_t(kStaticSorMaxPixels)];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
float* g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

// Device address of g_sor_scratch on the current device (looked up once).
float* scratch_for(int device) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[device]) {
        void* ptr = nullptr;
        AR_CUDA(cudaGetSymbolAddress(&ptr, g_sor_scratch));
        AR_CUDA(cudaDeviceGetAttribute(&g_num_sms[device], cudaDevAttrMultiProcessorCount, device));
        g_scratch_addr[device] = static_cast<float*>(ptr);
    }
    return g_scratch_addr[device];
}

}  // namespace

}  // namespace ar

using namespace ar;

extern "C" int ar_poisson_sor_static(const ar_integrator_cfg* cfg, uint32_t width, uint32_t height,
                                     const float* primal, const float* grad_x, const float* grad_y, float* out,
                                     void* cuda_stream) {
    return guarded([&] {
        AR_REQUIRE(cfg && primal && grad_x && grad_y && out, AR_ERR_INVALID_ARGUMENT, "null argument");
        AR_REQUIRE(cfg->poisson_solver == AR_POISSON_SOR, AR_ERR_UNSUPPORTED,
                   "ar_poisson_sor_static solves with red-black SOR only (cfg->poisson_solver must be AR_POISSON_SOR)");
        AR_REQUIRE(width > 0 && height > 0, AR_ERR_INVALID_ARGUMENT, "empty image");
        AR_REQUIRE(uint64_t(width) * height <= kStaticSorMaxPixels, AR_ERR_INVALID_ARGUMENT,
                   "image of " + std::to_string(uint64_t(width) * height) + " pixels exceeds the static scratch (" +
                       std::to_string(kStaticSorMaxPixels) + " pixels, AR_STATIC_SOR_MAX_PIXELS)");
        int device = 0;
        AR_CUDA(cudaGetDevice(&device));
        AR_REQUIRE(device >= 0 && device < kMaxDevices, AR_ERR_UNSUPPORTED, "device ordinal too large");
        require_device_ptr(primal, device, "primal");
        require_device_ptr(grad_x, device, "grad_x");
        require_device_ptr(grad_y, device, "grad_y");
        require_device_ptr(out, device, "out");
        float* scratch = scratch_for(device);
        float* rhs = scratch;
        float* img = scratch + 3 * size_t(kStaticSorMaxPixels);
        poisson_sor_with_scratch(static_cast<cudaStream_t>(cuda_stream), g_num_sms[device], *cfg, width, height,
                                 primal, grad_x, grad_y, rhs, img, out);
    });
}
