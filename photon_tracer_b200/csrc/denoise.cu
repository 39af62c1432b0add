// Edge-avoiding a-trous denoiser on the GPU: the filter of
// include/denoise.hpp:55-139 (demodulate by albedo, five 5x5 B3-spline passes
// with taps 1, 2, 4, 8, 16 apart, weights from normals, albedo and the
// variance-scaled luminance difference, variance filtered along), one thread
// per pixel per pass. Each pass reads a 5x5 neighbourhood of the previous
// pass's lighting, so the passes are separate launches ping-ponging two
// scratch buffers.
#include <cuda_runtime.h>

#include <string>

#include "../../include/photon_cuda.h"
#include "pt_host.hpp"

namespace {

__device__ __forceinline__ float lum(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }

__global__ void prepare(int n, const float* __restrict__ color, const float* __restrict__ albedo,
                        const float* __restrict__ normal, const float* __restrict__ variance, float* __restrict__ light,
                        float* __restrict__ var, float* __restrict__ nrm) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    for (int c = 0; c < 3; ++c) light[3 * p + c] = color[3 * p + c] / fmaxf(albedo[3 * p + c], 0.01f);
    const float a = fmaxf(lum(albedo[3 * p], albedo[3 * p + 1], albedo[3 * p + 2]), 0.01f);
    var[p] = fmaxf(variance[p], 0.0f) / (a * a);
    const float* s = normal + 3 * p;
    const float len = sqrtf(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (int c = 0; c < 3; ++c) nrm[3 * p + c] = len > 1e-6f ? s[c] / len : 0;
}

__global__ void atrous_pass(int w, int h, int step, const float* __restrict__ albedo, const float* __restrict__ nrm,
                            const float* __restrict__ light, const float* __restrict__ var,
                            float* __restrict__ light_next, float* __restrict__ var_next) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const float kernel[3] = {3.0f / 8, 1.0f / 4, 1.0f / 16};
    const size_t p = size_t(y) * w + x;
    const float np0 = nrm[3 * p], np1 = nrm[3 * p + 1], np2 = nrm[3 * p + 2];
    const float ap0 = albedo[3 * p], ap1 = albedo[3 * p + 1], ap2 = albedo[3 * p + 2];
    const bool p_sky = np0 == 0 && np1 == 0 && np2 == 0;
    const float lp = lum(light[3 * p], light[3 * p + 1], light[3 * p + 2]);
    float v = 0, vw = 0;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            const int qx = x + dx, qy = y + dy;
            if (qx < 0 || qy < 0 || qx >= w || qy >= h) continue;
            const float k = (dx ? 0.5f : 1) * (dy ? 0.5f : 1);
            v += k * var[size_t(qy) * w + qx];
            vw += k;
        }
    const float scale = 1 / (4.0f * sqrtf(v / vw) + 1e-4f);
    float s0 = 0, s1 = 0, s2 = 0, sum_w = 0, sum_var = 0;
    for (int dy = -2; dy <= 2; ++dy) {
        const int qy = y + dy * step;
        if (qy < 0 || qy >= h) continue;
        for (int dx = -2; dx <= 2; ++dx) {
            const int qx = x + dx * step;
            if (qx < 0 || qx >= w) continue;
            const size_t q = size_t(qy) * w + qx;
            const float nq0 = nrm[3 * q], nq1 = nrm[3 * q + 1], nq2 = nrm[3 * q + 2];
            const bool q_sky = nq0 == 0 && nq1 == 0 && nq2 == 0;
            if (p_sky != q_sky) continue;
            float weight = kernel[dx < 0 ? -dx : dx] * kernel[dy < 0 ? -dy : dy];
            if (!p_sky) {
                float nd = fmaxf(np0 * nq0 + np1 * nq1 + np2 * nq2, 0.0f);
                for (int k = 0; k < 6; ++k) nd *= nd;
                weight *= nd;
            }
            const float da0 = ap0 - albedo[3 * q], da1 = ap1 - albedo[3 * q + 1], da2 = ap2 - albedo[3 * q + 2];
            const float l0 = light[3 * q], l1 = light[3 * q + 1], l2 = light[3 * q + 2];
            weight *= expf(-(da0 * da0 + da1 * da1 + da2 * da2) * (1 / 0.01f) - fabsf(lp - lum(l0, l1, l2)) * scale);
            s0 += weight * l0;
            s1 += weight * l1;
            s2 += weight * l2;
            sum_w += weight;
            sum_var += weight * weight * var[q];
        }
    }
    light_next[3 * p] = s0 / sum_w;
    light_next[3 * p + 1] = s1 / sum_w;
    light_next[3 * p + 2] = s2 / sum_w;
    var_next[p] = sum_var / (sum_w * sum_w);
}

__global__ void finish(int n, const float* __restrict__ light, const float* __restrict__ albedo, float* __restrict__ out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    for (int c = 0; c < 3; ++c) out[3 * p + c] = light[3 * p + c] * fmaxf(albedo[3 * p + c], 0.01f);
}

pt_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PT_OK;
    return pt::fail(e == cudaErrorMemoryAllocation ? PT_ERR_OUT_OF_MEMORY : PT_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

size_t pt_denoise_atrous_scratch_floats(int width, int height) {
    if (width <= 0 || height <= 0) return 0;
    return 11 * size_t(width) * size_t(height);
}

pt_status pt_denoise_atrous_device(int w, int h, const float* color, const float* albedo, const float* normal,
                                   const float* variance, float* out, float* scratch, void* stream_) {
    pt::clear_error();
    if (w <= 0 || h <= 0) return pt::fail(PT_ERR_INVALID_ARG, "pt_denoise_atrous_device: bad size");
    if (!color || !albedo || !normal || !variance || !out || !scratch)
        return pt::fail(PT_ERR_INVALID_ARG, "pt_denoise_atrous_device: null pointer");
    if (size_t(w) * h > (size_t(1) << 30)) return pt::fail(PT_ERR_INVALID_ARG, "pt_denoise_atrous_device: too large");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    const int n = w * h;
    float* light = scratch;
    float* light_next = light + 3 * size_t(n);
    float* var = light_next + 3 * size_t(n);
    float* var_next = var + n;
    float* nrm = var_next + n;
    prepare<<<(n + 255) / 256, 256, 0, stream>>>(n, color, albedo, normal, variance, light, var, nrm);
    const dim3 block(16, 8), grid((w + 15) / 16, (h + 7) / 8);
    for (int pass = 0; pass < 5; ++pass) {
        atrous_pass<<<grid, block, 0, stream>>>(w, h, 1 << pass, albedo, nrm, light, var, light_next, var_next);
        float* t = light;
        light = light_next;
        light_next = t;
        t = var;
        var = var_next;
        var_next = t;
    }
    finish<<<(n + 255) / 256, 256, 0, stream>>>(n, light, albedo, out);
    return cuda_status(cudaGetLastError(), "pt_denoise_atrous_device");
}

pt_status pt_denoise_atrous(int w, int h, const float* color, const float* albedo, const float* normal,
                            const float* variance, float* out) {
    pt::clear_error();
    if (w <= 0 || h <= 0) return pt::fail(PT_ERR_INVALID_ARG, "pt_denoise_atrous: bad size");
    if (!color || !albedo || !normal || !variance || !out)
        return pt::fail(PT_ERR_INVALID_ARG, "pt_denoise_atrous: null pointer");
    const size_t n = size_t(w) * h;
    float* d = nullptr;
    const size_t floats = 3 * n * 4 + n + pt_denoise_atrous_scratch_floats(w, h);
    if (pt_status st = cuda_status(cudaMalloc(&d, floats * sizeof(float)), "pt_denoise_atrous: allocation")) return st;
    float *dc = d, *da = dc + 3 * n, *dn = da + 3 * n, *dv = dn + 3 * n, *dout = dv + n, *ds = dout + 3 * n;
    cudaError_t e = cudaMemcpy(dc, color, 3 * n * 4, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(da, albedo, 3 * n * 4, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(dn, normal, 3 * n * 4, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(dv, variance, n * 4, cudaMemcpyHostToDevice);
    pt_status st = cuda_status(e, "pt_denoise_atrous: copy");
    if (st == PT_OK) st = pt_denoise_atrous_device(w, h, dc, da, dn, dv, dout, ds, nullptr);
    if (st == PT_OK) st = cuda_status(cudaMemcpy(out, dout, 3 * n * 4, cudaMemcpyDeviceToHost), "pt_denoise_atrous: copy back");
    cudaFree(d);
    return st;
}

}  // extern "C"

// ---- the filter without any allocation ------------------------------------------------------
// Some callers of this library cannot call cudaMalloc: a host application that
// owns all device memory through its own pool and does not let plugins
// allocate, or a per-frame loop where an allocation -- which can synchronise
// the device and can fail under memory pressure -- is not allowed. For them
// pt_denoise_atrous_device_noalloc runs the same filter with its scratch in
// the array below, a fixed part of the library's device image: every GPU that
// loads the library holds these 11.5 MB until the process exits, and frames
// are limited to PT_ATROUS_NOALLOC_MAX_PIXELS pixels.
//
// Host code must not hand g_atrous_scratch to a kernel: here its name is only
// a host-side stand-in. The device address is looked up once per CUDA context,
// with that context current, by the first call in it (cudaGetSymbolAddress), so
// the first call on each device -- and the first after a cudaDeviceReset, which
// makes a new context where the module may load elsewhere -- should come
// before any stream capture. Every call
// uses the same array and leaves the last call's data in it; the filter writes
// every scratch value before reading it, so nothing needs clearing, but two
// calls whose work overlaps on the GPU (different streams, or different host
// threads on one device) race on the array and corrupt each other's output.
static __device__ __align__(256) float g_atrous_scratch[11 * size_t(PT_ATROUS_NOALLOC_MAX_PIXELS)];

#include <cuda.h>

#include <map>
#include <mutex>

namespace {
std::mutex g_scratch_lock;
// CUDA context id -> device address of g_atrous_scratch in that context. Keyed
// by context, not device ordinal: after a device reset the module is loaded
// again into a new context (a new id) and its address is looked up again.
std::map<unsigned long long, float*> g_scratch_addr;

// The id of the calling thread's current context (cuCtxGetId, CUDA 12), or 0
// when none is current yet. The driver calls are reached through the runtime's
// entry-point lookup, so the library needs no link against libcuda.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(p);
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}
}  // namespace

extern "C" pt_status pt_denoise_atrous_device_noalloc(int w, int h, const float* color, const float* albedo,
                                                      const float* normal, const float* variance, float* out,
                                                      void* stream) {
    pt::clear_error();
    if (w <= 0 || h <= 0) return pt::fail(PT_ERR_INVALID_ARG, "pt_denoise_atrous_device_noalloc: bad size");
    if (size_t(w) * size_t(h) > size_t(PT_ATROUS_NOALLOC_MAX_PIXELS))
        return pt::fail(PT_ERR_INVALID_ARG,
                        "pt_denoise_atrous_device_noalloc: " + std::to_string(w) + "x" + std::to_string(h) +
                            " is more than the " + std::to_string(PT_ATROUS_NOALLOC_MAX_PIXELS) +
                            " pixels its built-in scratch holds; use pt_denoise_atrous_device with your own scratch");
    if (!color || !albedo || !normal || !variance || !out)
        return pt::fail(PT_ERR_INVALID_ARG, "pt_denoise_atrous_device_noalloc: null pointer");
    float* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_lock);
        const unsigned long long ctx = current_context_id();
        auto it = ctx ? g_scratch_addr.find(ctx) : g_scratch_addr.end();
        if (it == g_scratch_addr.end()) {
            // Looking the symbol up also makes the device's primary context
            // current when no runtime call has yet on this thread.
            void* p = nullptr;
            if (pt_status st = cuda_status(cudaGetSymbolAddress(&p, g_atrous_scratch),
                                           "pt_denoise_atrous_device_noalloc: scratch address"))
                return st;
            scratch = static_cast<float*>(p);
            if (const unsigned long long now = current_context_id()) g_scratch_addr[now] = scratch;
        } else {
            scratch = it->second;
        }
    }
    return pt_denoise_atrous_device(w, h, color, albedo, normal, variance, out, scratch, stream);
}
