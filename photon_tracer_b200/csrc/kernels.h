// Launch interface between the host glue (api.cpp) and the kernels (*.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pt_layout.h"

struct PtCamDev {
    float origin[3], llc[3], horizontal[3], vertical[3];
};

// One render launch: scanlines [row0, row0 + rows) of a width x height image.
// Scanline j lands in output row (flip ? height - 1 - j : j - row0).
struct PtRenderParams {
    PtCamDev cam;
    int width, height, spp, depth;
    uint64_t seed;
    int first_sample;
    int rng_mode;               // PT_RNG_*
    int nee_ext;                // PT_FLAG_NEE_EXTENDED (megakernel, production streams)
    const uint64_t* states;     // PT_RNG_SNAPSHOT: per (pixel, sample) xoshiro state
    int row0, rows, flip;
    float* out;                 // 3 floats per pixel
    float* aux;                 // 7 floats per pixel or null
    unsigned long long* rays;   // one counter the launch adds its rays to (may be null)
    unsigned int* work;         // one zeroed work counter (megakernel)
};

// Sizing of persistent launches.
struct PtLaunchShape {
    int blocks, threads;
};

// Megakernel: persistent warps take pixels from a global counter; each lane
// renders its pixel's samples one path after another.
cudaError_t pt_launch_megakernel(const PtSceneDev& scene, const PtRenderParams& p, const PtLaunchShape& shape,
                                 cudaStream_t stream);
int pt_megakernel_blocks_per_sm(const PtSceneDev& scene, int threads, bool aux, bool snapshot, bool ext);

// Ray queries: closest hit (pt_hit records), any hit (bytes), and traversal
// work counters (5 x u64, added to).
cudaError_t pt_launch_trace_closest(const PtSceneDev& scene, const float* rays, size_t n, float tmin, float tmax,
                                    void* hits, cudaStream_t stream);
cudaError_t pt_launch_trace_any(const PtSceneDev& scene, const float* rays, size_t n, float tmin, float tmax,
                                uint8_t* occluded, cudaStream_t stream);
cudaError_t pt_launch_trace_count(const PtSceneDev& scene, const float* rays, size_t n, float tmin, float tmax,
                                  unsigned long long* counts, cudaStream_t stream);

// Distance to the first surface along each pixel's centre ray, top row first
// (0 on a miss).
cudaError_t pt_launch_primary_depth(const PtSceneDev& scene, const PtCamDev& cam, int width, int height, float* depth,
                                    cudaStream_t stream);

// Blocks of `threads` threads (and dyn_smem bytes of dynamic shared memory)
// of kernel fn that fit on one SM at once, from the device's limits and the
// kernel's registers and static shared memory.
int pt_resident_blocks(const void* fn, int threads, size_t dyn_smem);

// out[i] = float(sum[i] * inv): the mean of FP64 per-pixel sums.
cudaError_t pt_launch_mean_of_sum(const double* sum, size_t n, double inv, float* out, cudaStream_t stream);
