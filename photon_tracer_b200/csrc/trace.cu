// Ray-query kernels: closest hit and any hit for caller-supplied rays (one
// thread per ray), and the same closest-hit traversal instrumented to count
// the work the algorithmic-bytes roofline is defined on.
#include "../../include/photon_cuda.h"
#include "kernels.h"
#include "tracer.cuh"

using namespace ptd;

namespace {

__device__ __forceinline__ void load_ray(const float* rays, size_t i, V& o, V& d) {
    const float* r = rays + 6 * i;
    o = mk(r[0], r[1], r[2]);
    d = mk(r[3], r[4], r[5]);
}

// FLAT: scenes without instances take the one-traversal query (no
// instance-tree code in the kernel).
template <bool FLAT>
__global__ void __launch_bounds__(128) trace_closest_kernel(PtSceneDev S, const float* __restrict__ rays, size_t n,
                                                             float tmin, float tmax, pt_hit* __restrict__ hits) {
    PT_TRAV_STACK(stack, 128);
    bool overflow = false;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        V o, d;
        load_ray(rays, i, o, d);
        float t = tmax;
        Hit h;
        bool ok;
        if constexpr (FLAT) {
            ok = query_flat(S, o, d, tmin, t, false, h, stack);
        } else {
            Counts cnt;
            ok = closest<false>(S, o, d, tmin, t, h, stack, cnt);
        }
        if (!ok) {
            overflow = true;
            h.kind = PT_HIT_NONE;
        }
        uint32_t index, sub;
        resolve(S, h, index, sub);
        pt_hit out;
        out.kind = h.kind;
        out.index = h.kind == PT_HIT_NONE ? 0u : index;
        out.sub = sub;
        out.t = t;
        out.u = h.u;
        out.v = h.v;
        hits[i] = out;
    }
    if (overflow) atomicOr(S.status, PT_DEV_ERR_STACK);
}

template <bool FLAT>
__global__ void __launch_bounds__(128) trace_any_kernel(PtSceneDev S, const float* __restrict__ rays, size_t n,
                                                         float tmin, float tmax, uint8_t* __restrict__ occ) {
    PT_TRAV_STACK(stack, 128);
    bool overflow = false;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        V o, d;
        load_ray(rays, i, o, d);
        bool b;
        if constexpr (FLAT) {
            float t = tmax;
            Hit h;
            const bool ok = query_flat(S, o, d, tmin, t, true, h, stack);
            overflow |= !ok;
            b = ok && h.kind != PT_HIT_NONE;
        } else {
            Counts cnt;
            bool ovf = false;
            b = occluded<false>(S, o, d, tmin, tmax, stack, cnt, &ovf);
            overflow |= ovf;
        }
        occ[i] = b ? 1 : 0;
    }
    if (overflow) atomicOr(S.status, PT_DEV_ERR_STACK);
}

__global__ void __launch_bounds__(128) trace_count_kernel(PtSceneDev S, const float* __restrict__ rays, size_t n,
                                                           float tmin, float tmax,
                                                           unsigned long long* __restrict__ counts) {
    PT_TRAV_STACK(stack, 128);
    Counts cnt = {0, 0, 0, 0, 0};
    bool overflow = false;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        V o, d;
        load_ray(rays, i, o, d);
        float t = tmax;
        Hit h;
        if (!closest<true>(S, o, d, tmin, t, h, stack, cnt)) overflow = true;
    }
    unsigned long long v[5] = {cnt.nodes, cnt.order, cnt.tris, cnt.spheres, cnt.insts};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        unsigned long long x = v[k];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if ((threadIdx.x & 31) == 0) atomicAdd(counts + k, x);
    }
    if (overflow) atomicOr(S.status, PT_DEV_ERR_STACK);
}

// Distance to the first surface along each pixel's centre ray (the depth
// guide of the learned denoiser): u = (i + 0.5) / (W - 1), v = (j + 0.5) /
// (H - 1) on the camera of include/camera.hpp:39-47, scanline j stored in
// row H - 1 - j like the frame; 0 where the ray leaves the scene.
__global__ void __launch_bounds__(128) primary_depth_kernel(PtSceneDev S, PtCamDev C, int width, int height,
                                                             float* __restrict__ depth) {
    PT_TRAV_STACK(stack, 128);
    bool overflow = false;
    const V org = mk(C.origin[0], C.origin[1], C.origin[2]), llc = mk(C.llc[0], C.llc[1], C.llc[2]);
    const V hor = mk(C.horizontal[0], C.horizontal[1], C.horizontal[2]);
    const V ver = mk(C.vertical[0], C.vertical[1], C.vertical[2]);
    const size_t n = size_t(width) * height;
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        const int i = int(k % width), j = int(k / width);
        const float u = (float(i) + 0.5f) / float(width - 1), v = (float(j) + 0.5f) / float(height - 1);
        const V d = llc + hor * u + ver * v - org;
        float t = 1000.0f;
        Hit h;
        Counts cnt;
        if (!closest<false>(S, org, d, 0.001f, t, h, stack, cnt)) {
            overflow = true;
            h.kind = PT_HIT_NONE;
        }
        depth[size_t(height - 1 - j) * width + i] = h.kind == PT_HIT_NONE ? 0.0f : t * sqrtf(dot(d, d));
    }
    if (overflow) atomicOr(S.status, PT_DEV_ERR_STACK);
}

bool flat_scene(const PtSceneDev& S) { return S.inst_root == PT_NONE && S.n_instances == 0; }

int grid_for(size_t n, int threads) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t want = (n + threads - 1) / threads;
    const size_t cap = size_t(sms) * 16;
    return int(want < cap ? (want ? want : 1) : cap);
}

}  // namespace

cudaError_t pt_launch_trace_closest(const PtSceneDev& S, const float* rays, size_t n, float tmin, float tmax,
                                    void* hits, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    if (flat_scene(S))
        trace_closest_kernel<true><<<grid_for(n, 128), 128, 0, stream>>>(S, rays, n, tmin, tmax, static_cast<pt_hit*>(hits));
    else
        trace_closest_kernel<false><<<grid_for(n, 128), 128, 0, stream>>>(S, rays, n, tmin, tmax, static_cast<pt_hit*>(hits));
    return cudaGetLastError();
}

cudaError_t pt_launch_trace_any(const PtSceneDev& S, const float* rays, size_t n, float tmin, float tmax,
                                uint8_t* occ, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    if (flat_scene(S))
        trace_any_kernel<true><<<grid_for(n, 128), 128, 0, stream>>>(S, rays, n, tmin, tmax, occ);
    else
        trace_any_kernel<false><<<grid_for(n, 128), 128, 0, stream>>>(S, rays, n, tmin, tmax, occ);
    return cudaGetLastError();
}

cudaError_t pt_launch_trace_count(const PtSceneDev& S, const float* rays, size_t n, float tmin, float tmax,
                                  unsigned long long* counts, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    trace_count_kernel<<<grid_for(n, 128), 128, 0, stream>>>(S, rays, n, tmin, tmax, counts);
    return cudaGetLastError();
}

cudaError_t pt_launch_primary_depth(const PtSceneDev& S, const PtCamDev& cam, int width, int height, float* depth,
                                    cudaStream_t stream) {
    const size_t n = size_t(width) * height;
    if (n == 0) return cudaSuccess;
    primary_depth_kernel<<<grid_for(n, 128), 128, 0, stream>>>(S, cam, width, height, depth);
    return cudaGetLastError();
}
