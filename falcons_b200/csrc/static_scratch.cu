// Static device scratch for falcons_interp_decompress_noalloc (include/falcons_b200.h).
//
// Some callers cannot let a library allocate device memory.  An application that hands nearly all
// of HBM to its own pool at start-up (a simulation code, a training or serving framework) leaves
// cudaMalloc nothing to give, and a latency-bound decode thread cannot absorb cudaFree's implicit
// device-wide synchronisation or the first-use growth of a context's work buffers.  For those
// callers the scratch of the interpolation decompressor (one escape slot per code, per-tile escape
// counts and their prefix sums) lives here, in this module's static device memory: it is reserved
// when the module is loaded on a device and every later call on that device reuses it.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>

#include "../../include/falcons_b200.h"
#include "common.cuh"
#include "interp.cuh"
#include "static_scratch.cuh"

// One region per device (a __device__ variable has one instance per device the module is loaded on).
static __device__ __align__(256) unsigned char g_noalloc_scratch[FALCONS_NOALLOC_SCRATCH_BYTES];

namespace fb2 {
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_ptr[kMaxDevices];
}  // namespace

void *static_scratch_current_device() {
    int dev = -1;
    FB2_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw std::invalid_argument("device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        // Set-up, once per device, with that device current: resolving the symbol loads this
        // module (and so reserves the scratch) on the device, and the preload loads every
        // decompress kernel, so that no later call triggers a module or kernel load.
        void *p = nullptr;
        FB2_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        if (!p) throw cuda_error("static scratch has no device address");
        FB2_CUDA(interp_decompress_preload());
        g_scratch_ptr[dev] = p;
    }
    return g_scratch_ptr[dev];
}

}  // namespace fb2
