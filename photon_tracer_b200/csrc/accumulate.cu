// Ground truth accumulation: per-pixel radiance sums in FP64 across
// progressive passes. Each pass renders spp samples per pixel (continuing
// the per-pixel sample numbering through first_sample) into a float frame of
// averages; this kernel adds average * spp to the double sums, so the sum of
// millions of samples per pixel keeps its precision. This is the only FP64
// in the render path besides the reference's double-precision large-sphere
// test.
#include <cuda_runtime.h>

#include <string>

#include "../../include/photon_cuda.h"
#include "pt_host.hpp"

namespace {

__global__ void add_pass(size_t n, const float* __restrict__ frame, double weight, double* __restrict__ sum) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        sum[i] += double(frame[i]) * weight;
}

__global__ void mean_of_sum(size_t n, const double* __restrict__ sum, double inv, float* __restrict__ out) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = float(sum[i] * inv);
}

}  // namespace

cudaError_t pt_launch_mean_of_sum(const double* sum, size_t n, double inv, float* out, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const size_t blocks = (n + 255) / 256;
    mean_of_sum<<<unsigned(blocks < 148 * 32 ? blocks : 148 * 32), 256, 0, stream>>>(n, sum, inv, out);
    return cudaGetLastError();
}

extern "C" pt_status pt_accumulate_pass(const float* d_frame, size_t n_floats, double weight, double* d_sum,
                                        void* stream) {
    pt::clear_error();
    if (!d_frame || !d_sum) return pt::fail(PT_ERR_INVALID_ARG, "pt_accumulate_pass: null pointer");
    if (n_floats == 0) return PT_OK;
    const size_t blocks = (n_floats + 255) / 256;
    add_pass<<<unsigned(blocks < 148 * 32 ? blocks : 148 * 32), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        n_floats, d_frame, weight, d_sum);
    const cudaError_t e = cudaGetLastError();
    if (e) return pt::fail(PT_ERR_CUDA, std::string("pt_accumulate_pass: ") + cudaGetErrorString(e));
    return PT_OK;
}
