// ps_b200_prepare_particles_noalloc: ps_prepare_particles for callers that
// cannot allocate memory.
//
// The regular ps_prepare_particles creates a process-wide workspace on its
// first call (a stream, a device buffer for the per-block partial bounding
// boxes, a pinned result buffer, and device mirrors when the caller passes
// host arrays).  Some callers cannot allow that: an engine that reserves all
// device memory up front and forbids allocation inside its frame loop, so
// that a frame never stalls on the allocator or fails half-way for want of
// memory (the reference itself is built on the rule that the library never
// allocates, polesitter.h:20-24).  This entry point allocates nothing: its only
// scratch -- the partial boxes and the final box -- lives in the file-scope
// device array below, of fixed size, loaded with the library.
//
// Contract:
//   * x, y, z and out_morton_codes must be device memory; out_min_b,
//     out_max_b, out_range are host pointers (any may be NULL).
//   * cnt must be 1 .. kNoAllocMaxParticles (4,194,304); larger counts are
//     rejected with PS_EINVAL and a message in ps_b200_last_error().
//   * The first call on each device resolves the scratch array's device
//     address (cudaGetSymbolAddress) and caches it for that device.  The
//     cached address belongs to the device's context at that time: after
//     cudaDeviceReset the next call would pass a stale address, so do not
//     mix this entry point with device resets in one process.
//   * Work runs on the legacy default stream and the call returns after the
//     codes and the box are final.  All calls share the one scratch array, so
//     calls that overlap on the GPU (e.g. from several host threads) race;
//     serialise them.  Every call fully rewrites the scratch it reads, so
//     nothing needs clearing between calls.
#include <atomic>
#include <cstdio>

#include "psg_common.cuh"
#include "psg_kernels.h"

namespace psg {

constexpr int kNoAllocBlockParticles = 1024;
constexpr int kNoAllocMaxBlocks = 4096;
constexpr size_t kNoAllocMaxParticles = (size_t)kNoAllocBlockParticles * kNoAllocMaxBlocks;

// [0, kNoAllocMaxBlocks): one (min, max) per block of 1024 particles;
// [kNoAllocMaxBlocks, +2): the final (min, max) and (range, 1023/range).
// 32 KB + 16 B, held by every device that loads the library, until exit.
static __device__ __align__(256) float2 g_prepare_scratch[kNoAllocMaxBlocks + 2];

constexpr int kMaxDevices = 64;
static std::atomic<float2*> g_scratch_ptr[kMaxDevices];

static int scratch_on_current_device(float2** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PSG_EDEVICE;
    float2* p = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!p) {
        void* addr = nullptr;
        e = cudaGetSymbolAddress(&addr, g_prepare_scratch);
        if (e != cudaSuccess || !addr) return PSG_EDEVICE;
        p = static_cast<float2*>(addr);
        g_scratch_ptr[dev].store(p, std::memory_order_release);
    }
    *out = p;
    return PSG_OK;
}

static bool is_device_ptr(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace psg

extern "C" const char* psg_last_error(void);
extern "C" void psg_set_error(const char* msg);

extern "C" int psg_prepare_noalloc(const float* x, const float* y, const float* z, size_t n,
                                   uint32_t* codes, float* out_min, float* out_max,
                                   float* out_range, int variant) {
    using namespace psg;
    if (!x || !y || !z || !codes || n == 0) {
        psg_set_error("ps_b200_prepare_particles_noalloc: null array or zero count");
        return PSG_EINVAL;
    }
    if (n > kNoAllocMaxParticles) {
        char msg[160];
        std::snprintf(msg, sizeof(msg),
                      "ps_b200_prepare_particles_noalloc: %zu particles exceed its fixed "
                      "scratch (at most %zu)", n, kNoAllocMaxParticles);
        psg_set_error(msg);
        return PSG_EINVAL;
    }
    if (!is_device_ptr(x) || !is_device_ptr(y) || !is_device_ptr(z) || !is_device_ptr(codes)) {
        psg_set_error("ps_b200_prepare_particles_noalloc: x, y, z and the codes must be "
                      "device memory");
        return PSG_EINVAL;
    }
    float2* scratch = nullptr;
    int r = scratch_on_current_device(&scratch);
    if (r != PSG_OK) {
        psg_set_error("ps_b200_prepare_particles_noalloc: cudaGetSymbolAddress failed");
        return r;
    }
    const int grid = (int)((n + kNoAllocBlockParticles - 1) / kNoAllocBlockParticles);
    float* box = reinterpret_cast<float*>(scratch + kNoAllocMaxBlocks);
    launch_prepare(x, y, z, n, scratch, grid, codes, box, variant, (cudaStream_t)0);
    cudaError_t e = cudaGetLastError();
    float h[4] = {0.f, 0.f, 0.f, 0.f};
    if (e == cudaSuccess) e = cudaMemcpy(h, box, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        psg_set_error(cudaGetErrorString(e));
        return PSG_EDEVICE;
    }
    if (out_min) *out_min = h[0];
    if (out_max) *out_max = h[1];
    if (out_range) *out_range = h[2];
    return PSG_OK;
}
