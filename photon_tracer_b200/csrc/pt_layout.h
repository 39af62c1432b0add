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
    uint32_t n_spheres;       // top-level spheres
    int sky, sample_lights, use_bvh;
    int has_textures;         // some lambertian has a texture
    int ordered_boxes;        // every node child box has lo <= hi on each axis (no NaN)
};
