/*
 * Fixed scratch for sg_evaluate_device_noalloc.
 *
 * The evaluation sorts its query points before the walk and needs scratch
 * for that (keys, a histogram, the sorted coordinates and the permutation).
 * sg_evaluate_device grows a buffer with cudaMalloc for it; the no-allocation
 * entry point instead uses the array below, which every GPU that loads this
 * library holds until the process exits.
 *
 * In host code `g_noalloc_scratch` is only a host-side stand-in for the
 * device array, not a device address: a kernel given it would fault or, where
 * the GPU can reach host memory, use the wrong memory.  The device address is
 * obtained once per device with cudaGetSymbolAddress, with that device
 * current, and cached here; the cache entries are atomic, so host threads
 * may call concurrently.  A cudaDeviceReset ends every device allocation of
 * this library on that device, the cached address included: handles and
 * this cache do not survive it.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "sg_kernels.h"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[SG_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::atomic<void *> g_scratch_ptr[kMaxDevices];

} // namespace

extern "C" int sgk_noalloc_scratch(void **ptr, int64_t *bytes)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    void *p = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!p) {
        /* two threads may both look it up: they store the same address */
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev].store(p, std::memory_order_release);
    }
    *ptr = p;
    *bytes = SG_NOALLOC_SCRATCH_BYTES;
    return cudaSuccess;
}
