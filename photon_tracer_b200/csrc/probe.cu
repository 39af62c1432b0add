// Bandwidth probe for the traversal roofline (no counterpart in the
// reference). The traversal's node and primitive fetches are served from the
// 126 MB L2 when the scene fits there (the benchmark scenes do), so its
// roofline is reported against a measured L2 read rate as well as against
// the HBM copy rate: this kernel re-reads one L2-resident buffer `reps` times
// per launch with 16-byte loads that bypass L1 (ld.global.cg), every lane
// reading a coalesced stride of the buffer, so launch latency does not count.
#include <cuda_runtime.h>

#include "../../include/photon_cuda.h"
#include "pt_host.hpp"

namespace {

__global__ void __launch_bounds__(256) l2_read_kernel(const float4* __restrict__ p, size_t n4, int reps,
                                                      float* sink) {
    float acc = 0;
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    for (int r = 0; r < reps; ++r)
        for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n4; i += stride) {
            const float4 v = __ldcg(p + i);
            acc += (v.x + v.y) + (v.z + v.w);
        }
    // the sum is kept only so that the loads are not removed
    if (acc == -1.0f) sink[0] = acc;
}

}  // namespace

extern "C" pt_status pt_measure_l2_read(size_t bytes, int reps, double* gbs) {
    pt::clear_error();
    if (!gbs || bytes < 4096 || reps < 1) return pt::fail(PT_ERR_INVALID_ARG, "pt_measure_l2_read: bad argument");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t n4 = bytes / 16;
    void* buf = nullptr;
    if (cudaError_t e = cudaMalloc(&buf, n4 * 16 + 256)) return pt::fail(PT_ERR_OUT_OF_MEMORY, cudaGetErrorString(e));
    float* sink = reinterpret_cast<float*>(static_cast<char*>(buf) + n4 * 16);
    cudaStream_t s = nullptr;
    cudaEvent_t a = nullptr, z = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (!e) e = cudaEventCreate(&a);
    if (!e) e = cudaEventCreate(&z);
    if (!e) e = cudaMemsetAsync(buf, 0, n4 * 16, s);
    const int blocks = sms * 8;
    for (int k = 0; k < 3 && !e; ++k) {  // warm-up: the buffer into L2
        l2_read_kernel<<<blocks, 256, 0, s>>>(static_cast<const float4*>(buf), n4, reps, sink);
        e = cudaGetLastError();
    }
    if (!e) e = cudaEventRecord(a, s);
    for (int k = 0; k < 10 && !e; ++k) {
        l2_read_kernel<<<blocks, 256, 0, s>>>(static_cast<const float4*>(buf), n4, reps, sink);
        e = cudaGetLastError();
    }
    if (!e) e = cudaEventRecord(z, s);
    if (!e) e = cudaEventSynchronize(z);
    float ms = 0;
    if (!e) e = cudaEventElapsedTime(&ms, a, z);
    if (a) cudaEventDestroy(a);
    if (z) cudaEventDestroy(z);
    if (s) cudaStreamDestroy(s);
    cudaFree(buf);
    if (e) return pt::fail(PT_ERR_CUDA, std::string("pt_measure_l2_read: ") + cudaGetErrorString(e));
    *gbs = double(n4) * 16.0 * reps * 10 / (double(ms) / 1e3) / 1e9;
    return PT_OK;
}
