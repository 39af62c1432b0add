// The host-side image of the device arena (pt_layout.h), built by build_arena
// and uploaded as is.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <vector>

#include "pt_host.hpp"
#include "pt_layout.h"

namespace pt {

struct HostArena {
    std::vector<float> nodes;   // 32 floats per node
    std::vector<float> slots;   // 12 floats per slot
    std::vector<float> islots;  // 16 floats per instance slot
    std::vector<float4> large;
    std::vector<uint32_t> large_mat;
    std::vector<PtShadeSphere> sph;
    std::vector<PtShadeTri> tri;
    std::vector<PtShadeInst> inst;
    std::vector<PtMaterial> mat;
    std::vector<PtLight> lights;
    std::vector<PtTriLight> tri_lights;  // emissive flat triangles
    std::vector<float> light_cdf;        // extended pick: cumulative probabilities, spheres then triangles
    float pick_uniform = 0, pick_power = 0;
    std::vector<float> tri_uv;    // 6 per shading triangle
    std::vector<int4> tex;        // width, height, first texel float, 0
    std::vector<float> texels;    // linear RGB
    int has_textures = 0;
    uint32_t flat_root = PT_NONE, inst_root = PT_NONE;
    uint32_t n_flat_slots = 0, n_instances = 0, n_spheres = 0;
    uint32_t stack_entries = 0, max_depth = 0;
    int sky = 1, sample_lights = 1, use_bvh = 1;
};

pt_status build_arena(const pt_scene_desc& d, HostArena& A);

// 1 when every child box of every node (32 floats per node: lo[3][4],
// hi[3][4], first[4], count[4]) has lo <= hi on each axis, i.e. holds no NaN
// and is not inverted; the traversal's fast slab test relies on it.
int ordered_boxes(const std::vector<float>& nodes);
// 1 when every traversal stack entry of the scene's trees fits 8 bytes
// (PtSceneDev::stack_pack8): leaves of at most 15 primitives from below slot
// 2^26, node indices below 2^31.
int stack_pack8(const std::vector<float>& nodes);
// KiB of nodes and leaf slots (PtSceneDev::tree_kib), saturating.
uint32_t tree_kib(const std::vector<float>& nodes, const std::vector<float>& slots);

}  // namespace pt
