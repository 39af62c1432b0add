// Host-side internals of libphoton_cuda: error reporting, the BVH builder,
// transform helpers and the float vector arithmetic the scene generators use.
// Host code is compiled with -ffp-contract=off so every float expression
// rounds exactly as the reference's (which is built without FMA).
#pragma once
#include "../../include/photon_cuda.h"

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

namespace pt {

// ---- errors ------------------------------------------------------------------
void set_error(const std::string& msg);
void clear_error();
pt_status fail(pt_status code, const std::string& msg);

// ---- BVH and transforms (bvh_build.cpp) -----------------------------------------
void build_bvh(const float* boxes, uint32_t n, std::vector<pt_bvh_node>& nodes, std::vector<uint32_t>& order);
// The 4-wide collapse of a binary tree given per binary node its box (6
// floats), first (left child for interior nodes, leaf start otherwise) and
// count (0 for interior nodes); node 0 is the root.
void collapse_bvh(const float* boxes, const uint32_t* first, const uint32_t* count, uint32_t n_bin,
                  std::vector<pt_bvh_node>& nodes);
void triangle_box(const float p0[3], const float p1[3], const float p2[3], float out[6]);
void sphere_box(const float c[3], float r, float out[6]);
void affine_box(const pt_affine& x, const float in[6], float out[6]);
void affine_vector(const pt_affine& x, const float v[3], float out[3]);
void affine_point(const pt_affine& x, const float p[3], float out[3]);
pt_affine affine_inverse(const pt_affine& x);
uint32_t tree_depth(const std::vector<pt_bvh_node>& nodes, uint32_t root);
// The path-queue capacity of a scene's wavefront renders (0: the default,
// 2^20 paths in flight); the batch autotuner tries several.
void set_wave_slots(pt_scene* s, uint32_t slots);

// ---- float vector arithmetic, in the reference's evaluation order -------------------
// (include/vec3.hpp:58-118: dot is (x*x' + y*y') + z*z', normalize divides
// each component by the length, operator/ multiplies by the reciprocal)
struct V3 {
    float x, y, z;
};
inline V3 v3(float x, float y, float z) { return {x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, float t) { return {a.x * t, a.y * t, a.z * t}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 normalize(V3 a) {
    const float len = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return {a.x / len, a.y / len, a.z / len};
}
inline void store(float* d, V3 a) { d[0] = a.x; d[1] = a.y; d[2] = a.z; }
inline V3 load(const float* s) { return {s[0], s[1], s[2]}; }

// A triangle as the reference's constructors make it (include/triangle.hpp:26-35).
pt_triangle make_triangle(V3 a, V3 b, V3 c, uint32_t material);                       // flat
pt_triangle make_triangle(V3 a, V3 b, V3 c, V3 na, V3 nb, V3 nc, uint32_t material);  // smooth

}  // namespace pt
