// Resident blocks per SM of a kernel, computed from the device's limits and
// the kernel's own attributes (registers, static shared memory): the grid
// size of the persistent kernels.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"

namespace {

struct DeviceLimits {
    int smem_sm = 0, reserved = 0, threads_sm = 0, regs_sm = 0, blocks_sm = 0;
};

const DeviceLimits& limits() {
    static DeviceLimits devs[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    DeviceLimits& d = devs[dev];
    if (!d.threads_sm) {
        cudaDeviceGetAttribute(&d.smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&d.reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
        cudaDeviceGetAttribute(&d.regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&d.blocks_sm, cudaDevAttrMaxBlocksPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&d.threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    }
    return d;
}

}  // namespace

int pt_resident_blocks(const void* fn, int threads, size_t dyn_smem) {
    const DeviceLimits& d = limits();
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess || threads <= 0) return 1;
    // Registers are allocated per warp in units of 256 (8 per thread).
    const int regs = std::max(8, (fa.numRegs + 7) / 8 * 8);
    const int warps = (threads + 31) / 32;
    int n = d.blocks_sm > 0 ? d.blocks_sm : 32;
    if (d.threads_sm > 0) n = std::min(n, d.threads_sm / (warps * 32));
    if (d.regs_sm > 0) n = std::min(n, d.regs_sm / (regs * 32 * warps));
    const size_t smem = fa.sharedSizeBytes + dyn_smem + size_t(d.reserved);
    if (d.smem_sm > 0 && smem > 0) n = std::min<long>(n, long(size_t(d.smem_sm) / smem));
    return std::max(n, 1);
}
