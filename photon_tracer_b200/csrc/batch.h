// Launch interface of the batched renderer (batch.cu, batch.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pt_layout.h"

// One scene of a batch as the kernel sees it: its view of the merged arena
// (roots and ranges, all indices already rebased) and its frame.
struct PtBatchScene {
    uint32_t flat_root, inst_root;
    uint32_t large_base, n_large;
    uint32_t light_base, n_lights;
    uint32_t sky, sample_lights;
    uint32_t width, height, spp, depth;
    uint64_t seed;
    uint64_t out_offset;  // first float of its image in the batch output
    uint32_t tiles_x;     // 8x4 tiles per row of tiles
    uint32_t item_base;   // its first work item
    float cam[12];        // origin, lower-left corner, horizontal, vertical
};

struct PtBatchLaunch {
    const PtBatchScene* scenes;
    const PtSceneDev* views;           // per scene: the merged arena seen as that scene alone
    uint32_t n_scenes;
    uint32_t total_items;
    float* out;
    unsigned int* work;                // zeroed work counter
    unsigned int* done_pixels;         // per scene, zeroed
    unsigned long long* done_ns;       // per scene: global timer when its last pixel was written
    unsigned long long* start_ns;      // set to ~0 before the launch; the earliest block start
    unsigned long long* rays;          // added to (may be null)
    int any_instances;                 // some scene has an instance tree: the single-loop traversal
};

cudaError_t pt_launch_batch(const PtSceneDev& arena, const PtBatchLaunch& b, int threads, int sms,
                            cudaStream_t stream);
