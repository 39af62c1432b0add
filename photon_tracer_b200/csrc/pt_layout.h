// Device-side scene layout, shared by the host repack (scene.cpp) and the
// kernels. Everything a ray reads while traversing lives in a handful of flat
// arrays ("the arena"):
//
//   nodes      all 4-wide trees (flat, instance, every mesh), 128 B each, the
//              reference's bvh::node layout (include/bvh.hpp:27-32: lo[axis][child],
//              hi[axis][child], first[4], count[4]) with first[] rebased into the
//              arena. A leaf count word carries PT_LEAF_HAS_SPHERE in bit 31
//              when the leaf holds at least one sphere, and PT_LEAF_INSTANCES in
//              bit 30 for leaves of the instance tree.
//   slots      leaf entries in leaf order, 48 B each, so that a leaf's primitives
//              are contiguous and need no order[] indirection:
//                triangle: (p0.xyz, e1.x) (e1.yz, e2.xy) (e2.z, ref, 0, 0)
//                sphere:   (center.xyz, radius) (0) (0, ref | PT_SLOT_SPHERE, 0, 0)
//              ref is the primitive's original number (sphere or triangle
//              index; for a mesh tree, the triangle's index in its mesh).
//   islots     instance-tree leaf entries in leaf order, 64 B each:
//                to_object rows (m[r][0..2], t[r]) x3, (mesh root node, instance number, 0, 0)
//
// and shading data indexed by original numbers (read once per hit).
#pragma once
#include <math.h>
#include <stdint.h>

#define PT_LEAF_HAS_SPHERE 0x80000000u
#define PT_LEAF_INSTANCES 0x40000000u   // a leaf of the instance tree (entries are instance slots)
#define PT_COUNT_MASK 0x3fffffffu
#define PT_SLOT_SPHERE 0x80000000u
#define PT_NONE 0xffffffffu

// The traversal stack bound per ray. The reference bounds one tree walk by
// 3 * max_depth + 1 entries (include/bvh.hpp:66-68); scenes are checked at
// creation against the entries they can actually need.
#define PT_STACK_MAX 96

// Material flags.
#define PT_MF_EMITS 1u
#define PT_MF_DIFFUSE 2u
#define PT_MF_TRANSMISSIVE 4u

// Device error bits (scene status word).
#define PT_DEV_ERR_STACK 1u
#define PT_DEV_ERR_QUEUE 2u
#define PT_DEV_ERR_TIMEOUT 4u

#ifndef __CUDACC__
#include <vector_types.h>
#endif

struct PtMaterial {   // 48 B
    float4 albedo_type;   // albedo.xyz, type (as float bits of uint)
    float4 emission_fuzz; // emission.xyz, fuzz
    float4 ior_flags;     // ior, flags (bits), texture (bits; PT_NONE: none), 0
};

struct PtShadeTri {   // 64 B
    float4 n0_mat;  // n0.xyz, material (bits)
    float4 n1;
    float4 n2;
    float4 fn;      // face normal
};

struct PtShadeSphere {  // 32 B
    float4 cr;          // center.xyz, radius
    uint32_t mat, pad0, pad1, pad2;
};

struct PtShadeInst {  // 64 B
    float4 row[3];     // to_object rows (m[r][0..2], t[r])
    uint32_t tri_base; // first shading triangle of its mesh
    uint32_t material; // PT_NONE: keep the mesh's materials
    uint32_t mesh;
    uint32_t pad;
};

struct PtLight {   // 32 B: a light sphere with its emission
    float4 cr;
    float4 emission;
};

// An emissive triangle of the flat list, for the extended light sampling
// (PT_FLAG_NEE_EXTENDED): corner p0, edges, face normal, area, emission.
struct PtTriLight {  // 64 B
    float4 p0_area;  // p0.xyz, area
    float4 e1_er;    // e1.xyz, emission.x
    float4 e2_eg;    // e2.xyz, emission.y
    float4 fn_eb;    // face normal.xyz, emission.z
};

// The extended light choice: light i (spheres of the light list first, then
// the emissive triangles) is picked with probability
//   pick_uniform + pick_power * power_i,
// half uniform, half in proportion to power = luminance(emission) * area
// (4 pi r^2 for a sphere), the uniform half keeping every light reachable.
// Host and device compute power with these same float operations.
#if defined(__CUDACC__)
#define PT_HD __host__ __device__ __forceinline__
#else
#define PT_HD inline
#endif
PT_HD float pt_light_luminance(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }
PT_HD float pt_sphere_light_power(float lum, float radius) {
    const float p = lum * (4.0f * 3.14159265f * (radius * radius));
    return p > 0.0f && p < 3.0e38f ? p : 0.0f;
}
PT_HD float pt_triangle_area(float ax, float ay, float az, float bx, float by, float bz) {
    const float cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
    return 0.5f * sqrtf(cx * cx + cy * cy + cz * cz);
}
PT_HD float pt_triangle_light_power(float lum, float area) {
    const float p = lum * area;
    return p > 0.0f && p < 3.0e38f ? p : 0.0f;
}

// Everything a kernel needs, passed by value.
struct PtSceneDev {
    const float4* nodes;      // 8 float4 per node
    const float4* slots;      // 3 float4 per slot
    const float4* islots;     // 4 float4 per instance slot
    const float4* large;      // center, radius
    const uint32_t* large_mat;
    const PtShadeSphere* sph;
    const PtShadeTri* tri;
    const PtShadeInst* inst;
    const PtMaterial* mat;
    const PtLight* lights;
    const PtTriLight* tri_lights;  // emissive flat triangles (extended light sampling)
    const float* light_cdf;   // n_lights + n_tri_lights cumulative pick probabilities, last 1
    const float* tri_uv;      // 6 per shading triangle: texture coordinates at the corners
    const int4* tex;          // per texture: width, height, first texel float, 0
    const float* texels;      // linear RGB, 3 floats per texel, rows top first
    unsigned int* status;     // device error word
    uint32_t flat_root;       // PT_NONE when there is no flat tree
    uint32_t inst_root;
    uint32_t n_flat_slots;    // slots 0..n-1 are the flat primitives when !use_bvh
    uint32_t n_instances;
    uint32_t n_large;
    uint32_t n_lights;
    uint32_t n_tri_lights;
    float pick_uniform, pick_power;  // the extended pick probability of a light of power p: u + w * p
    uint32_t n_spheres;       // top-level spheres
    int sky, sample_lights, use_bvh;
    int has_textures;         // some lambertian has a texture
    int ordered_boxes;        // every node child box has lo <= hi on each axis (no NaN)
    int stack_pack8;          // every leaf holds <= 15 entries from below slot 2^26 and every
                              // node index is below 2^31: flat-tree stack entries fit 8 bytes
    uint32_t tree_kib;        // nodes and leaf slots of every tree, KiB (saturating)
};
