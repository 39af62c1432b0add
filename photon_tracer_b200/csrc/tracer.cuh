// Device side of the render hot path: BVH4 traversal, sphere and triangle
// intersection, hit records, the Sobol/xoshiro sampler and the materials.
//
// Every float expression is written in the reference's evaluation order and
// this file is compiled with -fmad=false -prec-div=true -prec-sqrt=true, so
// closest hits (primitive, t, u, v) are bit-identical to the reference's
// geometry::hit on the same rays. The comments cite the reference function
// each routine restates (photon_tracer, include/...).
#pragma once

#include <type_traits>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/photon_cuda.h"
#include "pt_layout.h"

namespace ptd {

// ---- float3 helpers in the reference's order (include/vec3.hpp:71-118) --------------
struct V {
    float x, y, z;
};
__host__ __device__ __forceinline__ V mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V operator-(V a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V operator*(V a, V b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V operator*(V a, float t) { return {a.x * t, a.y * t, a.z * t}; }
__device__ __forceinline__ float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V cross(V a, V b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// vec3::normalize divides each component by the length (vec3.hpp:95-98).
__device__ __forceinline__ V normalize(V a) {
    const float len = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
    return {a.x / len, a.y / len, a.z / len};
}
// vec3::operator/ multiplies by the reciprocal (vec3.hpp:87-89).
__device__ __forceinline__ V div(V a, float t) { return a * (1.0f / t); }

// sinf and cosf of one angle through sincosf: one argument reduction for
// both, and the same two values (checked bit for bit on the GPU for every
// float in [-2 pi, 2 pi], the range the samplers pass).
__device__ __forceinline__ void sin_cos(float x, float& s, float& c) { sincosf(x, &s, &c); }
__device__ __forceinline__ V xyz(float4 f) { return {f.x, f.y, f.z}; }

// SSE minps / maxps (include/simd4.hpp:15-16): the second operand unless the
// first compares strictly less / greater, which also decides NaNs.
__device__ __forceinline__ float sse_min(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float sse_max(float a, float b) { return a > b ? a : b; }

__device__ __forceinline__ uint32_t fbits(float f) { return __float_as_uint(f); }

// ---- hits --------------------------------------------------------------------------------
struct Hit {
    uint32_t kind;   // PT_HIT_*
    uint32_t index;  // slot (flat / mesh) or large sphere number, resolved later
    uint32_t inst;   // instance number for instance hits
    float u, v;
};

// Work counters for the algorithmic-bytes roofline (nodes, leaf entries,
// triangles, spheres, instances).
struct Counts {
    uint32_t nodes, order, tris, spheres, insts;
};

struct StackEntry {
    uint32_t first, count;
    float t;
    uint32_t pad;
};

// ---- the traversal stack -----------------------------------------------------------------
// Entries a traversal pushes and pops (bvh.hpp:67-103: node or leaf, entry
// distance). Each thread's entries [0, SH) live in shared memory, entries
// [SH, PT_STACK_MAX) in a per-thread local array. The shared part is laid out
// [depth][thread] in 16-byte entries: the lanes of a warp touch consecutive
// 16-byte words whatever depth each lane is at, so a 128-bit access is free
// of bank conflicts, and it is reached through a 32-bit shared-window address
// (ld/st.shared, no generic-address check). Walks of the benchmark trees
// rarely go deeper than SH, so their pushes and pops stay in shared memory;
// the local array (L1-cached) takes only the deep tail, and every push is
// still checked against PT_STACK_MAX. Measured with identical results: 8
// entries speed the wavefront stages up 5% and the closest-hit queries 2-3%
// (4 entries: +3% / +1%; 16: slower); kernels that keep other per-lane state
// in shared memory choose their own count (the megakernel: 0).
#ifndef PT_SH_STACK
#define PT_SH_STACK 8
#endif

#ifndef PT_SH_STACK_ASM
#define PT_SH_STACK_ASM 1
#endif

template <int SH, int NT>
struct TravStack {
#if PT_SH_STACK_ASM
    uint32_t base;      // shared-window address of this thread's entry 0
#else
    uint4* col;         // this thread's entry 0 in the block's shared array
#endif
    StackEntry* deep;   // PT_STACK_MAX entries; only [SH, PT_STACK_MAX) are used
    __device__ __forceinline__ void put(int i, StackEntry e) {
        if (SH > 0 && i < SH) {
#if PT_SH_STACK_ASM
            asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(base + uint32_t(i) * (16u * NT)),
                         "r"(e.first), "r"(e.count), "r"(__float_as_uint(e.t)), "r"(e.pad));
#else
            col[i * NT] = make_uint4(e.first, e.count, __float_as_uint(e.t), e.pad);
#endif
        } else {
            deep[i] = e;
        }
    }
    __device__ __forceinline__ StackEntry get(int i) const {
        if (SH > 0 && i < SH) {
#if PT_SH_STACK_ASM
            uint32_t f, c, t, p;
            asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                         : "=r"(f), "=r"(c), "=r"(t), "=r"(p)
                         : "r"(base + uint32_t(i) * (16u * NT)));
            return {f, c, __uint_as_float(t), p};
#else
            const uint4 q = col[i * NT];
            return {q.x, q.y, __uint_as_float(q.z), q.w};
#endif
        }
        return deep[i];
    }
};

// Declares `name`, the traversal stack of the calling thread, in a kernel of
// NT threads per block with SH entries per thread in shared memory: the
// block's shared part and this thread's local array.
#if PT_SH_STACK_ASM
#define PT_TRAV_STACK_BASE(arr) static_cast<uint32_t>(__cvta_generic_to_shared(&arr[threadIdx.x]))
#else
#define PT_TRAV_STACK_BASE(arr) (&arr[threadIdx.x])
#endif
#define PT_TRAV_STACK_N(name, NT, SH)                                                        \
    __shared__ uint4 name##_shared[(SH) > 0 ? (SH) * (NT) : 1];                               \
    StackEntry name##_deep[PT_STACK_MAX];                                                     \
    ::ptd::TravStack<(SH), (NT)> name{PT_TRAV_STACK_BASE(name##_shared), name##_deep}
#define PT_TRAV_STACK(name, NT) PT_TRAV_STACK_N(name, NT, PT_SH_STACK)

// The same stack in 8-byte entries, for walks of one flat tree whose leaves
// all hold at most 15 primitives starting below slot 2^26 (PtSceneDev::
// stack_pack8, checked when the scene is uploaded; the binned SAH builder
// keeps leaves at <= 8 primitives except at its depth limit). An entry is
// (word, t): an interior node is its index (bit 31 clear); a leaf sets bit
// 31, carries PT_LEAF_HAS_SPHERE in bit 30, its count in bits 26-29 and its
// first slot in bits 0-25. Half the bytes per entry: the shared part takes
// 8 bytes per entry and thread ([depth][thread], a warp's 64-bit accesses
// are conflict-free at any per-lane depth) and the local tail 768 bytes per
// thread instead of 1,536.
__device__ __forceinline__ uint32_t pack8_word(uint32_t first, uint32_t count) {
    return count == 0 ? first
                      : (0x80000000u | ((count & PT_LEAF_HAS_SPHERE) >> 1) | ((count & 15u) << 26) | first);
}
__device__ __forceinline__ StackEntry unpack8(uint32_t w, uint32_t t) {
    if (w & 0x80000000u) return {w & 0x03ffffffu, ((w >> 26) & 15u) | ((w << 1) & PT_LEAF_HAS_SPHERE), __uint_as_float(t), 0u};
    return {w, 0u, __uint_as_float(t), 0u};
}

template <int SH, int NT>
struct PackedStack {
    uint32_t base;  // shared-window address of this thread's entry 0
    uint2* deep;    // PT_STACK_MAX entries; only [SH, PT_STACK_MAX) are used
    __device__ __forceinline__ void put(int i, StackEntry e) {
        const uint32_t w = pack8_word(e.first, e.count), t = __float_as_uint(e.t);
        if (SH > 0 && i < SH) {
            asm volatile("st.shared.v2.u32 [%0], {%1, %2};" ::"r"(base + uint32_t(i) * (8u * NT)), "r"(w), "r"(t));
        } else {
            deep[i] = make_uint2(w, t);
        }
    }
    __device__ __forceinline__ StackEntry get(int i) const {
        if (SH > 0 && i < SH) {
            uint32_t w, t;
            asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(w), "=r"(t) : "r"(base + uint32_t(i) * (8u * NT)));
            return unpack8(w, t);
        }
        const uint2 q = deep[i];
        return unpack8(q.x, q.y);
    }
};

// Declares `name`, the traversal stack of the calling thread in a kernel of
// form TREES with NT threads per block: 8-byte entries, SH8 of them in shared
// memory, in the PT_TREES_FLAT8 form; 16-byte entries, SH16 in shared memory,
// otherwise.
#define PT_FORM_STACK(name, TREES, NT, SH16, SH8)                                                      \
    constexpr bool name##_pack = (TREES) == ::ptd::PT_TREES_FLAT8;                                    \
    constexpr int name##_sh16 = name##_pack ? 0 : (SH16), name##_sh8 = name##_pack ? (SH8) : 0;       \
    __shared__ uint4 name##_s16[name##_sh16 > 0 ? name##_sh16 * (NT) : 1];                            \
    __shared__ uint2 name##_s8[name##_sh8 > 0 ? name##_sh8 * (NT) : 1];                               \
    std::conditional_t<name##_pack, uint2, ::ptd::StackEntry> name##_deep[PT_STACK_MAX];              \
    std::conditional_t<name##_pack, ::ptd::PackedStack<name##_sh8, (NT)>,                             \
                       ::ptd::TravStack<name##_sh16, (NT)>>                                           \
        name{static_cast<uint32_t>(__cvta_generic_to_shared(name##_pack ? static_cast<void*>(&name##_s8[0])  \
                                                                        : static_cast<void*>(&name##_s16[0]))) + \
                 threadIdx.x * (name##_pack ? 8u : 16u),                                                \
             name##_deep}

// ---- primitives ------------------------------------------------------------------------
// sphere::intersect<float> (include/sphere.hpp:25-48).
__device__ __forceinline__ bool sphere_hit(float4 cr, V o, V d, float t_min, float& t_max) {
    const float ox = o.x - cr.x, oy = o.y - cr.y, oz = o.z - cr.z;
    const float a = d.x * d.x + d.y * d.y + d.z * d.z;
    const float half_b = ox * d.x + oy * d.y + oz * d.z;
    const float c = ox * ox + oy * oy + oz * oz - cr.w * cr.w;
    const float disc = half_b * half_b - a * c;
    if (disc < 0) return false;
    const float sqrtd = sqrtf(disc);
    float root = (-half_b - sqrtd) / a;
    if (root < t_min || root > t_max) {
        root = (-half_b + sqrtd) / a;
        if (root < t_min || root > t_max) return false;
    }
    t_max = root;
    return true;
}

// sphere::intersect<double> (include/sphere.hpp:25-48 with P = double), the
// test geometry::hit and occluded use for large spheres (include/geometry.hpp:117-118,
// 157-160). The only double arithmetic in the traversal: it is what makes the
// t of a ray bouncing off a radius-1000 ground exact.
__device__ __forceinline__ bool sphere_hit_double(float4 cr, V o, V d, float t_min, float& t_max) {
    const double ox = double(o.x) - double(cr.x), oy = double(o.y) - double(cr.y), oz = double(o.z) - double(cr.z);
    const double dx = d.x, dy = d.y, dz = d.z;
    const double a = dx * dx + dy * dy + dz * dz;
    const double half_b = ox * dx + oy * dy + oz * dz;
    const double c = ox * ox + oy * oy + oz * oz - double(cr.w) * double(cr.w);
    const double disc = half_b * half_b - a * c;
    if (disc < 0) return false;
    const double sqrtd = sqrt(disc);
    double root = (-half_b - sqrtd) / a;
    if (root < double(t_min) || root > double(t_max)) {
        root = (-half_b + sqrtd) / a;
        if (root < double(t_min) || root > double(t_max)) return false;
    }
    t_max = float(root);
    return true;
}

// triangle::intersect, Moller-Trumbore (include/triangle.hpp:40-61). The slot
// holds (p0, e1.x) (e1.yz, e2.xy) (e2.z, ...).
__device__ __forceinline__ bool tri_hit(float4 a, float4 b, float4 c, V o, V d, float t_min, float& t_max,
                                        float& u_out, float& v_out) {
    const V p0 = mk(a.x, a.y, a.z), e1 = mk(a.w, b.x, b.y), e2 = mk(b.z, b.w, c.x);
    const V pvec = cross(d, e2);
    const float det = dot(e1, pvec);
    if (fabsf(det) < 1e-12f) return false;
    const float inv_det = 1.0f / det;
    const V tvec = o - p0;
    const float u = dot(tvec, pvec) * inv_det;
    if (u < 0 || u > 1) return false;
    const V qvec = cross(tvec, e1);
    const float v = dot(d, qvec) * inv_det;
    if (v < 0 || u + v > 1) return false;
    const float t = dot(e2, qvec) * inv_det;
    if (t < t_min || t > t_max) return false;
    t_max = t;
    u_out = u;
    v_out = v;
    return true;
}

// affine::vector / point (include/transform.hpp:15-20) with rows (m[r][0..2], t[r]).
__device__ __forceinline__ V aff_vector(const float4 r[3], V v) {
    return {r[0].x * v.x + r[0].y * v.y + r[0].z * v.z, r[1].x * v.x + r[1].y * v.y + r[1].z * v.z,
            r[2].x * v.x + r[2].y * v.y + r[2].z * v.z};
}
__device__ __forceinline__ V aff_point(const float4 r[3], V p) { return aff_vector(r, p) + mk(r[0].w, r[1].w, r[2].w); }
// affine::transposed (include/transform.hpp:23-27).
__device__ __forceinline__ V aff_transposed(const float4 r[3], V v) {
    return {r[0].x * v.x + r[1].x * v.y + r[2].x * v.z, r[0].y * v.x + r[1].y * v.y + r[2].y * v.z,
            r[0].z * v.x + r[1].z * v.y + r[2].z * v.z};
}

// ---- BVH4 traversal (include/bvh.hpp:57-106) ---------------------------------------------
// Pops an entry; skips it when t >= t_max; a leaf calls leaf(first, count);
// a node is slab-tested against [t_min, t_max] for its four children, and the
// children hit are pushed farthest first, equal entry distances in child
// order (a stable sort by descending t), so the nearest is popped next --
// the same visiting order as the reference, which decides equal-t ties.
// Returns false if the stack would overflow (the ray is then abandoned).
//
// Three ways of doing the same arithmetic faster, each exact:
//  * PT_TRAV_KEEP_NEAREST: the entry that would be popped next (the nearest
//    child) stays in registers instead of a push and a pop; it still gets
//    the pruning test. Off by default: it measured slower (the megakernel
//    lost 18% on the 1024x1024 room frame, 1.5% on pure ray queries).
//  * PT_TRAV_FAST_MINMAX: the reference's SSE minps/maxps return the second
//    operand when either is NaN, which PTX min/max (NaN-ignoring) do not. A
//    slab value (lo - o) * (1/d) can only be NaN when 1/d is infinite or
//    zero, or o is not finite (inf - inf, 0 * inf), and the t_max clamp only
//    when t_max is NaN. For rays with finite, nonzero inverse directions and
//    a finite origin, while t_max is not NaN, no operand is NaN and the two
//    forms agree (a -0/+0 difference cannot change any comparison the
//    traversal makes), so those nodes use the one-instruction min/max; other
//    rays keep the exact emulation. The node boxes must be NaN-free too
//    (PtSceneDev::ordered_boxes: lo <= hi for every child and axis, which
//    the empty-child encoding lo = hi = +inf also meets). Then, with the
//    sign of each inverse direction known, (lo - o) * inv <= (hi - o) * inv
//    or the reverse holds for every child (rounding is monotonic), so the
//    per-axis min / max is the value from the near plane / far plane: fast
//    rays load the near planes where the emulation reads lo and skip the
//    six per-axis min / max of each child.
//  * PT_TRAV_F32X2: the six subtractions and six multiplications of two
//    children's slabs are issued as packed pairs (sub/mul.rn.f32x2), which
//    round each lane exactly as the scalar instructions do.
#ifndef PT_TRAV_KEEP_NEAREST
#define PT_TRAV_KEEP_NEAREST 0
#endif
#ifndef PT_TRAV_FAST_MINMAX
#define PT_TRAV_FAST_MINMAX 1
#endif
#ifndef PT_TRAV_F32X2
#define PT_TRAV_F32X2 1
#endif

__device__ __forceinline__ bool finite_nonzero(float x) { return fabsf(x) < __int_as_float(0x7f800000) && x != 0.0f; }
__device__ __forceinline__ bool finite_f(float x) { return fabsf(x) < __int_as_float(0x7f800000); }

// (a - b) * c on two lanes at once, rounded per lane like the scalar form.
__device__ __forceinline__ float2 sub_mul2(float2 a, float2 b, float2 c) {
    unsigned long long ua, ub, uc, r;
    ua = (unsigned long long)__float_as_uint(a.x) | ((unsigned long long)__float_as_uint(a.y) << 32);
    ub = (unsigned long long)__float_as_uint(b.x) | ((unsigned long long)__float_as_uint(b.y) << 32);
    uc = (unsigned long long)__float_as_uint(c.x) | ((unsigned long long)__float_as_uint(c.y) << 32);
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(ua), "l"(ub));
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(r), "l"(uc));
    return make_float2(__uint_as_float(unsigned(r)), __uint_as_float(unsigned(r >> 32)));
}

// Position of each hit child among the hit children after a stable sort by
// descending entry distance: child c lands after those strictly farther and
// after equal ones with a smaller child number (position n - 1 is popped
// next). Each of the six pairs is decided once, missed children keyed at
// -inf so that they never move a hit child (entry distances are at least
// t_min, never -inf or NaN). Against counting, per child, the three others
// ahead of it: same positions, +2.5% on the room frame together with
// sin_cos.
__device__ __forceinline__ void child_ranks(const float (&tn)[4], int mask, int (&rank)[4]) {
    float key[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        key[c] = (mask & (1 << c)) ? tn[c] : -__int_as_float(0x7f800000);
        rank[c] = 0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int c = k + 1; c < 4; ++c) {
            if (key[k] >= key[c]) ++rank[c];
            else ++rank[k];
        }
}

template <bool COUNT, class Stack, class Leaf>
__device__ __forceinline__ bool traverse(const PtSceneDev& S, uint32_t root, V o, V d, float t_min, float& t_max,
                                         Stack& stack, int base, Counts& cnt, Leaf&& leaf) {
    const float4* __restrict__ nodes = S.nodes;
    const float ix = 1.0f / d.x, iy = 1.0f / d.y, iz = 1.0f / d.z;
    const bool ray_fast = PT_TRAV_FAST_MINMAX && S.ordered_boxes && finite_nonzero(ix) && finite_nonzero(iy) &&
                          finite_nonzero(iz) && finite_f(o.x) && finite_f(o.y) && finite_f(o.z) && t_min == t_min;
    // float4 index of each axis' near plane (lo: 0-2, hi: 3-5); the far
    // plane is the other one.
    const int nx = ray_fast && ix < 0 ? 3 : 0, ny = ray_fast && iy < 0 ? 4 : 1, nz = ray_fast && iz < 0 ? 5 : 2;
    int top = base;
    uint32_t cf = root, cc = 0;
    float ct = t_min;
    bool have = true;
    if (!PT_TRAV_KEEP_NEAREST) {
        stack.put(top++, {root, 0u, t_min, 0u});
        have = false;
    }
    while (true) {
        if (!have) {
            if (top == base) break;
            const StackEntry e = stack.get(--top);
            cf = e.first;
            cc = e.count;
            ct = e.t;
        }
        have = false;
        if (ct >= t_max) continue;
        if (cc != 0) {
            if (!leaf(cf, cc, top)) return false;
            continue;
        }
        const float4* nd = nodes + 8 * size_t(cf);
        const float4 lox = __ldg(nd + nx), loy = __ldg(nd + ny), loz = __ldg(nd + nz);
        const float4 hix = __ldg(nd + (3 - nx)), hiy = __ldg(nd + (5 - ny)), hiz = __ldg(nd + (7 - nz));
        const uint4 first = __ldg(reinterpret_cast<const uint4*>(nd + 6));
        const uint4 count = __ldg(reinterpret_cast<const uint4*>(nd + 7));
        if (COUNT) cnt.nodes++;
        // Slab values per child: x0 = (lo.x - o.x) * ix ... z1 = (hi.z - o.z) * iz
        // (for fast rays lo / hi are the near / far planes).
        float X0[4], X1[4], Y0[4], Y1[4], Z0[4], Z1[4];
        if (PT_TRAV_F32X2) {
            const float2 ox = make_float2(o.x, o.x), oy = make_float2(o.y, o.y), oz = make_float2(o.z, o.z);
            const float2 vx = make_float2(ix, ix), vy = make_float2(iy, iy), vz = make_float2(iz, iz);
#define PT_PAIR(ARR, V4, O2, I2)                                       \
    {                                                                  \
        const float2 a = sub_mul2(make_float2(V4.x, V4.y), O2, I2);    \
        const float2 b = sub_mul2(make_float2(V4.z, V4.w), O2, I2);    \
        ARR[0] = a.x; ARR[1] = a.y; ARR[2] = b.x; ARR[3] = b.y;        \
    }
            PT_PAIR(X0, lox, ox, vx)
            PT_PAIR(X1, hix, ox, vx)
            PT_PAIR(Y0, loy, oy, vy)
            PT_PAIR(Y1, hiy, oy, vy)
            PT_PAIR(Z0, loz, oz, vz)
            PT_PAIR(Z1, hiz, oz, vz)
#undef PT_PAIR
        } else {
            const float lx[4] = {lox.x, lox.y, lox.z, lox.w}, hx[4] = {hix.x, hix.y, hix.z, hix.w};
            const float ly[4] = {loy.x, loy.y, loy.z, loy.w}, hy[4] = {hiy.x, hiy.y, hiy.z, hiy.w};
            const float lz[4] = {loz.x, loz.y, loz.z, loz.w}, hz[4] = {hiz.x, hiz.y, hiz.z, hiz.w};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                X0[c] = (lx[c] - o.x) * ix;
                X1[c] = (hx[c] - o.x) * ix;
                Y0[c] = (ly[c] - o.y) * iy;
                Y1[c] = (hy[c] - o.y) * iy;
                Z0[c] = (lz[c] - o.z) * iz;
                Z1[c] = (hz[c] - o.z) * iz;
            }
        }
        float tn[4];
        int mask = 0;
        if (ray_fast && t_max == t_max) {
            // near plane values are each axis' minimum (lo <= hi, sign of
            // the inverse direction known): no per-axis min / max
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const float n_ = fmaxf(fmaxf(X0[c], Y0[c]), fmaxf(Z0[c], t_min));
                const float f_ = fminf(fminf(X1[c], Y1[c]), fminf(Z1[c], t_max));
                tn[c] = n_;
                mask |= (n_ <= f_) ? (1 << c) : 0;
            }
        } else {
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const float n_ = sse_max(sse_max(sse_min(X0[c], X1[c]), sse_min(Y0[c], Y1[c])),
                                         sse_max(sse_min(Z0[c], Z1[c]), t_min));
                const float f_ = sse_min(sse_min(sse_max(X0[c], X1[c]), sse_max(Y0[c], Y1[c])),
                                         sse_min(sse_max(Z0[c], Z1[c]), t_max));
                tn[c] = n_;
                mask |= (n_ <= f_) ? (1 << c) : 0;
            }
        }
        if (mask == 0) continue;
        const int n = __popc(mask);
        const int kept = PT_TRAV_KEEP_NEAREST ? 1 : 0;
        if (top + n - kept > PT_STACK_MAX) return false;
        const uint32_t fs[4] = {first.x, first.y, first.z, first.w};
        const uint32_t cs[4] = {count.x, count.y, count.z, count.w};
        // Position of child c among the hit children after a stable sort by
        // descending entry distance: those strictly farther, plus equal ones
        // with a smaller child number. Position n-1 is visited next.
        int rank[4];
        child_ranks(tn, mask, rank);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (!(mask & (1 << c))) continue;
            const int pos = rank[c];
            if (PT_TRAV_KEEP_NEAREST && pos == n - 1) {
                cf = fs[c];
                cc = cs[c];
                ct = tn[c];
            } else {
                stack.put(top + pos, {fs[c], cs[c], tn[c], 0u});
            }
        }
        top += n - kept;
        have = PT_TRAV_KEEP_NEAREST;
    }
    return true;
}

// ---- one loop over all trees ---------------------------------------------------------------
// The scene queries below walk the flat tree, then the instance tree, and for
// every instance in an instance leaf that instance's mesh tree, in exactly
// the order geometry::hit / occluded do (include/geometry.hpp:111-190), but
// in ONE loop over one stack: entering an instance pushes a "resume the
// leaf at the next instance" entry, a "back to the world ray" entry and the
// mesh root, and switches the ray to object space. Neither marker is pruned
// (a leaf's instances are all visited, as in the reference). One copy of the
// node and leaf code per query kind instead of one per tree: +44% on the
// 10,000-instance scene's megakernel frame. Scenes without instances keep the
// per-tree loop, which is tighter for a single tree (the one loop lost
// 11-26% there). Also measured and rejected: a "while-while" form (inner
// nodes until every lane holds a leaf, then leaves): -17% megakernel,
// -27% ray queries on the room.
#ifndef PT_TRAV_UNIFIED
#define PT_TRAV_UNIFIED 1
#endif

enum : uint32_t { PT_ENT_NODE = 0u, PT_ENT_RESUME = 1u, PT_ENT_WORLD = 2u };

struct TravRay {
    V o, d;
    float ix, iy, iz;
    bool fast;
    int nx, ny, nz;  // float4 index of each axis' near plane (lo: 0-2, hi: 3-5)
    __device__ __forceinline__ void set(V o_, V d_, float t_min, bool ordered) {
        o = o_;
        d = d_;
        ix = 1.0f / d.x;
        iy = 1.0f / d.y;
        iz = 1.0f / d.z;
        fast = PT_TRAV_FAST_MINMAX && ordered && finite_nonzero(ix) && finite_nonzero(iy) && finite_nonzero(iz) &&
               finite_f(o.x) && finite_f(o.y) && finite_f(o.z) && t_min == t_min;
        nx = fast && ix < 0 ? 3 : 0;
        ny = fast && iy < 0 ? 4 : 1;
        nz = fast && iz < 0 ? 5 : 2;
    }
};

// Slab-tests node cf's four children against [t_min, t_max] and pushes the
// ones hit, farthest first (bvh.hpp:72-103). False if the stack would overflow.
template <bool COUNT, class Stack>
__device__ __forceinline__ bool expand_node(const float4* __restrict__ nodes, uint32_t cf, const TravRay& r,
                                            float t_min, float t_max, Stack& stack, int& top, Counts& cnt) {
    const float4* nd = nodes + 8 * size_t(cf);
    const float4 lox = __ldg(nd + r.nx), loy = __ldg(nd + r.ny), loz = __ldg(nd + r.nz);
    const float4 hix = __ldg(nd + (3 - r.nx)), hiy = __ldg(nd + (5 - r.ny)), hiz = __ldg(nd + (7 - r.nz));
    const uint4 first = __ldg(reinterpret_cast<const uint4*>(nd + 6));
    const uint4 count = __ldg(reinterpret_cast<const uint4*>(nd + 7));
    if (COUNT) cnt.nodes++;
    float X0[4], X1[4], Y0[4], Y1[4], Z0[4], Z1[4];
    {
        const float2 ox = make_float2(r.o.x, r.o.x), oy = make_float2(r.o.y, r.o.y), oz = make_float2(r.o.z, r.o.z);
        const float2 vx = make_float2(r.ix, r.ix), vy = make_float2(r.iy, r.iy), vz = make_float2(r.iz, r.iz);
#define PT_PAIR(ARR, V4, O2, I2)                                       \
    {                                                                  \
        const float2 a = sub_mul2(make_float2(V4.x, V4.y), O2, I2);    \
        const float2 b = sub_mul2(make_float2(V4.z, V4.w), O2, I2);    \
        ARR[0] = a.x; ARR[1] = a.y; ARR[2] = b.x; ARR[3] = b.y;        \
    }
        PT_PAIR(X0, lox, ox, vx)
        PT_PAIR(X1, hix, ox, vx)
        PT_PAIR(Y0, loy, oy, vy)
        PT_PAIR(Y1, hiy, oy, vy)
        PT_PAIR(Z0, loz, oz, vz)
        PT_PAIR(Z1, hiz, oz, vz)
#undef PT_PAIR
    }
    float tn[4];
    int mask = 0;
    if (r.fast && t_max == t_max) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float n_ = fmaxf(fmaxf(X0[c], Y0[c]), fmaxf(Z0[c], t_min));
            const float f_ = fminf(fminf(X1[c], Y1[c]), fminf(Z1[c], t_max));
            tn[c] = n_;
            mask |= (n_ <= f_) ? (1 << c) : 0;
        }
    } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float n_ = sse_max(sse_max(sse_min(X0[c], X1[c]), sse_min(Y0[c], Y1[c])),
                                     sse_max(sse_min(Z0[c], Z1[c]), t_min));
            const float f_ = sse_min(sse_min(sse_max(X0[c], X1[c]), sse_max(Y0[c], Y1[c])),
                                     sse_min(sse_max(Z0[c], Z1[c]), t_max));
            tn[c] = n_;
            mask |= (n_ <= f_) ? (1 << c) : 0;
        }
    }
    if (mask == 0) return true;
    const int n = __popc(mask);
    if (top + n > PT_STACK_MAX) return false;
    const uint32_t fs[4] = {first.x, first.y, first.z, first.w};
    const uint32_t cs[4] = {count.x, count.y, count.z, count.w};
    // Stable sort by descending entry distance: child c lands after those
    // strictly farther and after equal ones with a smaller child number.
    int rank[4];
    child_ranks(tn, mask, rank);
#pragma unroll
    for (int c = 0; c < 4; ++c)
        if (mask & (1 << c)) stack.put(top + rank[c], {fs[c], cs[c], tn[c], PT_ENT_NODE});
    top += n;
    return true;
}

// The BVH part of geometry::hit (ANY = false: nearest hit into h and t_max)
// or of geometry::occluded (ANY = true: stops at the first blocker).
// Returns bit 0 on stack overflow, bit 1 when (ANY) something blocks.
template <bool COUNT, bool ANY, class Stack>
__device__ __forceinline__ int walk(const PtSceneDev& S, V wo, V wd, float t_min, float& t_max, Hit& h,
                                    Stack& stack, Counts& cnt) {
    TravRay r;
    r.set(wo, wd, t_min, S.ordered_boxes);
    uint32_t cur_inst = 0;
    bool in_mesh = false;
    int top = 0;
    if (S.inst_root != PT_NONE) stack.put(top++, {S.inst_root, 0u, t_min, PT_ENT_NODE});
    if (S.flat_root != PT_NONE) stack.put(top++, {S.flat_root, 0u, t_min, PT_ENT_NODE});
    while (top > 0) {
        const StackEntry e = stack.get(--top);
        uint32_t k = e.first, end = 0;
        if (e.pad == PT_ENT_WORLD) {
            r.set(wo, wd, t_min, S.ordered_boxes);
            in_mesh = false;
            continue;
        }
        if (e.pad == PT_ENT_RESUME) {
            end = e.count;
        } else {
            if (e.t >= t_max) continue;
            if (e.count == 0) {
                if (!expand_node<COUNT>(S.nodes, e.first, r, t_min, t_max, stack, top, cnt)) return 1;
                continue;
            }
            if (!(e.count & PT_LEAF_INSTANCES)) {
                // A leaf of primitive slots: the flat tree's (triangles and
                // spheres) or, inside an instance, its mesh's (triangles).
                const uint32_t n = e.count & PT_COUNT_MASK;
                const bool spheres = (e.count & PT_LEAF_HAS_SPHERE) != 0;
                for (uint32_t q = e.first; q < e.first + n; ++q) {
                    const float4* sl = S.slots + 3 * size_t(q);
                    if (COUNT) cnt.order++;
                    const float4 c = __ldg(sl + 2);
                    float tt = t_max, u, v;
                    float& tref = ANY ? tt : t_max;
                    bool hit;
                    bool sph = spheres && (fbits(c.y) & PT_SLOT_SPHERE);
                    if (sph) {
                        if (COUNT) cnt.spheres++;
                        hit = sphere_hit(__ldg(sl), r.o, r.d, t_min, tref);
                    } else {
                        if (COUNT) cnt.tris++;
                        hit = tri_hit(__ldg(sl), __ldg(sl + 1), c, r.o, r.d, t_min, tref, u, v);
                    }
                    if (!hit) continue;
                    if (ANY) return 2;
                    if (in_mesh) {
                        h.kind = PT_HIT_INSTANCE;
                        h.index = q;
                        h.inst = cur_inst;
                        h.u = u;
                        h.v = v;
                    } else if (sph) {
                        h.kind = PT_HIT_SPHERE;
                        h.index = q;
                    } else {
                        h.kind = PT_HIT_TRIANGLE;
                        h.index = q;
                        h.u = u;
                        h.v = v;
                    }
                }
                continue;
            }
            end = e.first + (e.count & PT_COUNT_MASK);
        }
        // Enter instance k of an instance leaf [.., end) (hit_instance, :212-229).
        if (k >= end) continue;
        if (top + 3 > PT_STACK_MAX) return 1;
        const float4* is = S.islots + 4 * size_t(k);
        const float4 rows[3] = {__ldg(is), __ldg(is + 1), __ldg(is + 2)};
        const uint4 meta = __ldg(reinterpret_cast<const uint4*>(is + 3));
        if (COUNT) {
            cnt.order++;
            cnt.insts++;
        }
        if (k + 1 < end) stack.put(top++, {k + 1, end, -__int_as_float(0x7f800000), PT_ENT_RESUME});
        stack.put(top++, {0u, 0u, -__int_as_float(0x7f800000), PT_ENT_WORLD});
        stack.put(top++, {meta.x, 0u, t_min, PT_ENT_NODE});
        r.set(aff_point(rows, wo), aff_vector(rows, wd), t_min, S.ordered_boxes);
        cur_inst = meta.y;
        in_mesh = true;
    }
    return 0;
}

// ---- the scene queries ---------------------------------------------------------------------
// geometry::hit (include/geometry.hpp:111-152) up to the choice of the
// nearest primitive: large spheres in double, then the flat tree, then the
// instance tree whose leaves walk each mesh's tree with the ray moved into
// object space (hit_instance, :212-229). Returns false on stack overflow.
// Which traversal form the scene queries compile: PT_TREES_EACH one loop
// per tree (the tighter form for a flat tree alone), PT_TREES_ONE the single
// loop over all trees (walk; faster with instances), PT_TREES_AUTO both,
// picked per scene (instances present -> walk). The megakernel is built in
// the two single forms and the host launches the one for its scene, so a
// flat scene's kernel carries no two-level code.
// PT_TREES_FLAT: scenes without instances; no instance-tree code at all.
// PT_TREES_FLAT8: a kernel form, not a query form -- PT_TREES_FLAT with the
// traversal stack in 8-byte entries (PackedStack); the kernel passes
// PT_TREES_FLAT to the queries.
enum { PT_TREES_AUTO = 0, PT_TREES_EACH = 1, PT_TREES_ONE = 2, PT_TREES_FLAT = 3, PT_TREES_FLAT8 = 4 };

template <bool COUNT, int TREES = PT_TREES_AUTO, class Stack>
__device__ __forceinline__ bool closest(const PtSceneDev& S, V o, V d, float t_min, float& t_max, Hit& h,
                                        Stack& stack, Counts& cnt) {
    h.kind = PT_HIT_NONE;
    h.index = 0;
    h.inst = 0;
    h.u = 0;
    h.v = 0;
    for (uint32_t i = 0; i < S.n_large; ++i)
        if (sphere_hit_double(__ldg(S.large + i), o, d, t_min, t_max)) {
            h.kind = PT_HIT_LARGE;
            h.index = i;
        }

    // One leaf of the flat tree: slots [first, first + count).
    auto flat_leaf = [&](uint32_t first, uint32_t count_word, int) -> bool {
        const uint32_t count = count_word & PT_COUNT_MASK;
        const bool spheres = (count_word & PT_LEAF_HAS_SPHERE) != 0;
        for (uint32_t k = first; k < first + count; ++k) {
            const float4* s = S.slots + 3 * size_t(k);
            if (COUNT) cnt.order++;
            if (spheres) {
                const float4 c = __ldg(s + 2);
                if (fbits(c.y) & PT_SLOT_SPHERE) {
                    if (COUNT) cnt.spheres++;
                    if (sphere_hit(__ldg(s), o, d, t_min, t_max)) {
                        h.kind = PT_HIT_SPHERE;
                        h.index = k;
                    }
                    continue;
                }
                if (COUNT) cnt.tris++;
                if (tri_hit(__ldg(s), __ldg(s + 1), c, o, d, t_min, t_max, h.u, h.v)) {
                    h.kind = PT_HIT_TRIANGLE;
                    h.index = k;
                }
            } else {
                if (COUNT) cnt.tris++;
                if (tri_hit(__ldg(s), __ldg(s + 1), __ldg(s + 2), o, d, t_min, t_max, h.u, h.v)) {
                    h.kind = PT_HIT_TRIANGLE;
                    h.index = k;
                }
            }
        }
        return true;
    };

    // One leaf of the instance tree: each instance walks its mesh's tree on
    // the stack above the current top.
    auto inst_leaf = [&](uint32_t first, uint32_t count_word, int top) -> bool {
        const uint32_t count = count_word & PT_COUNT_MASK;
        for (uint32_t k = first; k < first + count; ++k) {
            const float4* is = S.islots + 4 * size_t(k);
            float4 rows[3] = {__ldg(is), __ldg(is + 1), __ldg(is + 2)};
            const uint4 meta = __ldg(reinterpret_cast<const uint4*>(is + 3));
            if (COUNT) { cnt.order++; cnt.insts++; }
            const V lo = aff_point(rows, o), ld = aff_vector(rows, d);
            bool found = false;
            uint32_t slot = 0;
            float u = h.u, v = h.v;
            auto mesh_leaf = [&](uint32_t f, uint32_t cw, int) -> bool {
                const uint32_t c = cw & PT_COUNT_MASK;
                for (uint32_t q = f; q < f + c; ++q) {
                    const float4* s = S.slots + 3 * size_t(q);
                    if (COUNT) { cnt.order++; cnt.tris++; }
                    if (tri_hit(__ldg(s), __ldg(s + 1), __ldg(s + 2), lo, ld, t_min, t_max, u, v)) {
                        found = true;
                        slot = q;
                    }
                }
                return true;
            };
            if (!traverse<COUNT>(S, meta.x, lo, ld, t_min, t_max, stack, top, cnt, mesh_leaf)) return false;
            if (found) {
                h.kind = PT_HIT_INSTANCE;
                h.index = slot;
                h.inst = meta.y;
                h.u = u;
                h.v = v;
            }
        }
        return true;
    };

    if constexpr (TREES == PT_TREES_FLAT) {
        if (S.use_bvh) {
            if (S.flat_root != PT_NONE)
                if (!traverse<COUNT>(S, S.flat_root, o, d, t_min, t_max, stack, 0, cnt, flat_leaf)) return false;
        } else if (S.n_flat_slots) {
            flat_leaf(0, S.n_flat_slots | PT_LEAF_HAS_SPHERE, 0);
        }
        return true;
    }
    if (S.use_bvh) {
#if PT_TRAV_UNIFIED
        if constexpr (TREES != PT_TREES_EACH)
            if (TREES == PT_TREES_ONE || S.inst_root != PT_NONE)
                return !(walk<COUNT, false>(S, o, d, t_min, t_max, h, stack, cnt) & 1);
#endif
        if (S.flat_root != PT_NONE)
            if (!traverse<COUNT>(S, S.flat_root, o, d, t_min, t_max, stack, 0, cnt, flat_leaf)) return false;
        if (S.inst_root != PT_NONE)
            if (!traverse<COUNT>(S, S.inst_root, o, d, t_min, t_max, stack, 0, cnt, inst_leaf)) return false;
    } else {
        // Without the BVH every primitive, then every instance, in order (:135-139).
        if (S.n_flat_slots) flat_leaf(0, S.n_flat_slots | PT_LEAF_HAS_SPHERE, 0);
        if (S.n_instances)
            if (!inst_leaf(0, S.n_instances, 0)) return false;
    }
    return true;
}

// geometry::occluded (include/geometry.hpp:156-190): whether anything lies on
// the ray within [t_min, t_max]. Stops at the first blocker, which is where
// the reference's traversal stops doing work too (it collapses t_far to t_min).
// *overflow is set when a stack would overflow.
template <bool COUNT, int TREES = PT_TREES_AUTO, class Stack>
__device__ __forceinline__ bool occluded(const PtSceneDev& S, V o, V d, float t_min, float t_max,
                                         Stack& stack, Counts& cnt, bool* overflow) {
    for (uint32_t i = 0; i < S.n_large; ++i) {
        float t = t_max;
        if (sphere_hit_double(__ldg(S.large + i), o, d, t_min, t)) return true;
    }
    bool blocked = false;
    float t_far = t_max;
    auto flat_leaf = [&](uint32_t first, uint32_t count_word, int) -> bool {
        const uint32_t count = count_word & PT_COUNT_MASK;
        const bool spheres = (count_word & PT_LEAF_HAS_SPHERE) != 0;
        for (uint32_t k = first; k < first + count && !blocked; ++k) {
            const float4* s = S.slots + 3 * size_t(k);
            float t = t_far, u, v;
            if (COUNT) cnt.order++;
            const float4 c = __ldg(s + 2);
            if (spheres && (fbits(c.y) & PT_SLOT_SPHERE)) {
                if (COUNT) cnt.spheres++;
                blocked = sphere_hit(__ldg(s), o, d, t_min, t);
            } else {
                if (COUNT) cnt.tris++;
                blocked = tri_hit(__ldg(s), __ldg(s + 1), c, o, d, t_min, t, u, v);
            }
        }
        if (blocked) t_far = t_min;
        return true;
    };
    auto inst_leaf = [&](uint32_t first, uint32_t count_word, int top) -> bool {
        const uint32_t count = count_word & PT_COUNT_MASK;
        for (uint32_t k = first; k < first + count && !blocked; ++k) {
            const float4* is = S.islots + 4 * size_t(k);
            float4 rows[3] = {__ldg(is), __ldg(is + 1), __ldg(is + 2)};
            const uint4 meta = __ldg(reinterpret_cast<const uint4*>(is + 3));
            if (COUNT) { cnt.order++; cnt.insts++; }
            const V lo = aff_point(rows, o), ld = aff_vector(rows, d);
            float t_mesh = t_far;
            bool found = false;
            auto mesh_leaf = [&](uint32_t f, uint32_t cw, int) -> bool {
                const uint32_t c = cw & PT_COUNT_MASK;
                for (uint32_t q = f; q < f + c && !found; ++q) {
                    const float4* s = S.slots + 3 * size_t(q);
                    float u, v;
                    if (COUNT) { cnt.order++; cnt.tris++; }
                    if (tri_hit(__ldg(s), __ldg(s + 1), __ldg(s + 2), lo, ld, t_min, t_mesh, u, v)) {
                        found = true;
                        t_mesh = t_min;
                    }
                }
                return true;
            };
            if (!traverse<COUNT>(S, meta.x, lo, ld, t_min, t_mesh, stack, top, cnt, mesh_leaf)) return false;
            blocked = found;
        }
        if (blocked) t_far = t_min;
        return true;
    };
    if constexpr (TREES == PT_TREES_FLAT) {
        if (S.use_bvh) {
            if (S.flat_root != PT_NONE &&
                !traverse<COUNT>(S, S.flat_root, o, d, t_min, t_far, stack, 0, cnt, flat_leaf)) {
                *overflow = true;
                return false;
            }
        } else if (S.n_flat_slots) {
            flat_leaf(0, S.n_flat_slots | PT_LEAF_HAS_SPHERE, 0);
        }
        return blocked;
    }
    if (S.use_bvh) {
#if PT_TRAV_UNIFIED
        if constexpr (TREES != PT_TREES_EACH) {
            if (TREES == PT_TREES_ONE || S.inst_root != PT_NONE) {
                Hit unused;
                const int res = walk<COUNT, true>(S, o, d, t_min, t_far, unused, stack, cnt);
                if (res & 1) {
                    *overflow = true;
                    return false;
                }
                return (res & 2) != 0;
            }
        }
#endif
        if (S.flat_root != PT_NONE)
            if (!traverse<COUNT>(S, S.flat_root, o, d, t_min, t_far, stack, 0, cnt, flat_leaf)) {
                *overflow = true;
                return false;
            }
        if (!blocked && S.inst_root != PT_NONE) {
            t_far = t_max;
            if (!traverse<COUNT>(S, S.inst_root, o, d, t_min, t_far, stack, 0, cnt, inst_leaf)) {
                *overflow = true;
                return false;
            }
        }
    } else {
        if (S.n_flat_slots) flat_leaf(0, S.n_flat_slots | PT_LEAF_HAS_SPHERE, 0);
        if (!blocked && S.n_instances) {
            t_far = t_max;
            if (!inst_leaf(0, S.n_instances, 0)) {
                *overflow = true;
                return false;
            }
        }
    }
    return blocked;
}

// closest (any = false) and occluded (any = true) for a scene without
// instances, through ONE traversal: a kernel that issues both kinds of query
// from one call site carries one copy of the node and leaf code, and lanes
// on a shadow ray traverse alongside lanes on a path ray. The any-hit form
// stops at the first blocker (h.kind set), the point where occluded stops
// doing work; until then both forms run the same tests with the same t_max,
// so each returns what closest / occluded return. False when the stack
// would overflow.
template <class Stack>
__device__ __forceinline__ bool query_flat(const PtSceneDev& S, V o, V d, float t_min, float& t_max, bool any,
                                           Hit& h, Stack& stack) {
    h.kind = PT_HIT_NONE;
    h.index = 0;
    h.inst = 0;
    h.u = 0;
    h.v = 0;
    for (uint32_t i = 0; i < S.n_large; ++i)
        if (sphere_hit_double(__ldg(S.large + i), o, d, t_min, t_max)) {
            h.kind = PT_HIT_LARGE;
            h.index = i;
            if (any) return true;
        }
    // false stops the traversal: only after an any-hit blocker.
    auto leaf = [&](uint32_t first, uint32_t count_word, int) -> bool {
        const uint32_t count = count_word & PT_COUNT_MASK;
        const bool spheres = (count_word & PT_LEAF_HAS_SPHERE) != 0;
        for (uint32_t k = first; k < first + count; ++k) {
            const float4* s = S.slots + 3 * size_t(k);
            const float4 c = __ldg(s + 2);
            bool hit;
            if (spheres && (fbits(c.y) & PT_SLOT_SPHERE)) {
                hit = sphere_hit(__ldg(s), o, d, t_min, t_max);
                if (hit) h.kind = PT_HIT_SPHERE;
            } else {
                hit = tri_hit(__ldg(s), __ldg(s + 1), c, o, d, t_min, t_max, h.u, h.v);
                if (hit) h.kind = PT_HIT_TRIANGLE;
            }
            if (hit) {
                h.index = k;
                if (any) return false;
            }
        }
        return true;
    };
    Counts cnt;
    if (S.use_bvh) {
        if (S.flat_root != PT_NONE && !traverse<false>(S, S.flat_root, o, d, t_min, t_max, stack, 0, cnt, leaf))
            return any && h.kind != PT_HIT_NONE;
    } else if (S.n_flat_slots) {
        leaf(0, S.n_flat_slots | PT_LEAF_HAS_SPHERE, 0);
    }
    return true;
}

// The original primitive number of a closest hit (for ray queries).
__device__ __forceinline__ void resolve(const PtSceneDev& S, const Hit& h, uint32_t& index, uint32_t& sub) {
    index = h.index;
    sub = 0;
    if (h.kind == PT_HIT_SPHERE || h.kind == PT_HIT_TRIANGLE) {
        index = fbits(__ldg(S.slots + 3 * size_t(h.index) + 2).y) & ~PT_SLOT_SPHERE;
    } else if (h.kind == PT_HIT_INSTANCE) {
        index = h.inst;
        sub = fbits(__ldg(S.slots + 3 * size_t(h.index) + 2).y);
    }
}

// ---- hit records (include/hittable.hpp:7-21) -------------------------------------------------
struct Rec {
    V p, normal;
    float t;
    bool front_face;
    bool sampled_light;
    uint32_t mat;
    float tex_u, tex_v;  // texture coordinates (only filled in scenes with textures)
    // Extended light sampling only: which light was hit (0 none, 1 a light
    // sphere: lgeo = center, radius; 2 an emissive flat triangle: lgeo = face
    // normal, area), for the light-sampling density of the hit direction.
    uint32_t lkind;
    float4 lgeo;
};

// sphere::fill (include/sphere.hpp:50-58)
__device__ __forceinline__ void fill_sphere(float4 cr, uint32_t mat, V o, V d, float t, Rec& rec) {
    rec.t = t;
    rec.p = o + d * t;
    const V outward = (rec.p - xyz(cr)) * (1.0f / cr.w);
    rec.front_face = dot(d, outward) < 0;
    rec.normal = rec.front_face ? outward : -outward;
    rec.mat = mat;
}

// triangle::fill (include/triangle.hpp:63-74), direction d in the triangle's space.
template <bool TEX>
__device__ __forceinline__ void fill_triangle(const PtSceneDev& S, uint32_t g, V d, float u, float v, Rec& rec) {
    const PtShadeTri* __restrict__ tri = S.tri;
    const float4 a = __ldg(&tri[g].n0_mat), b = __ldg(&tri[g].n1), c = __ldg(&tri[g].n2), f = __ldg(&tri[g].fn);
    rec.front_face = dot(d, xyz(f)) < 0;
    const float w = 1 - u - v;
    const V n = normalize(xyz(a) * w + xyz(b) * u + xyz(c) * v);
    rec.normal = rec.front_face ? n : -n;
    rec.mat = fbits(a.w);
    if (TEX && S.has_textures) {  // rec.tex_u, tex_v (:72-73)
        const float* q = S.tri_uv + 6 * size_t(g);
        rec.tex_u = __ldg(q) * w + __ldg(q + 2) * u + __ldg(q + 4) * v;
        rec.tex_v = __ldg(q + 1) * w + __ldg(q + 3) * u + __ldg(q + 5) * v;
    }
}

// image_texture::sample (include/texture.hpp:25-33): bilinear, repeating
// outside [0, 1), v up the image while rows are stored top first.
__device__ __forceinline__ V texel(const PtSceneDev& S, int4 t, int x, int y) {
    x = ((x % t.x) + t.x) % t.x;
    y = ((y % t.y) + t.y) % t.y;
    const float* p = S.texels + size_t(uint32_t(t.z)) + 3 * (size_t(y) * size_t(t.x) + size_t(x));
    return mk(__ldg(p), __ldg(p + 1), __ldg(p + 2));
}
__device__ __forceinline__ V sample_texture(const PtSceneDev& S, uint32_t k, float u, float v) {
    const int4 t = __ldg(S.tex + k);
    const float x = (u - floorf(u)) * float(t.x) - 0.5f;
    const float y = (1 - (v - floorf(v))) * float(t.y) - 0.5f;
    const int x0 = static_cast<int>(floorf(x)), y0 = static_cast<int>(floorf(y));
    const float fx = x - float(x0), fy = y - float(y0);
    return texel(S, t, x0, y0) * ((1 - fx) * (1 - fy)) + texel(S, t, x0 + 1, y0) * (fx * (1 - fy)) +
           texel(S, t, x0, y0 + 1) * ((1 - fx) * fy) + texel(S, t, x0 + 1, y0 + 1) * (fx * fy);
}

// The record geometry::hit fills for the nearest primitive (:141-151,
// fill_instance :234-244).
// TEX = false compiles out the texture coordinates (kernels for scenes
// without textures: two fewer live registers through the shading code).
template <bool TEX = true, bool EXT = false>
__device__ __forceinline__ void fill(const PtSceneDev& S, const Hit& h, V o, V d, float t, Rec& rec) {
    rec.sampled_light = false;
    if (EXT) rec.lkind = 0;
    rec.t = t;
    rec.tex_u = 0;
    rec.tex_v = 0;
    switch (h.kind) {
        case PT_HIT_LARGE:
            fill_sphere(__ldg(S.large + h.index), __ldg(S.large_mat + h.index), o, d, t, rec);
            break;
        case PT_HIT_SPHERE: {
            const uint32_t i = fbits(__ldg(S.slots + 3 * size_t(h.index) + 2).y) & ~PT_SLOT_SPHERE;
            const float4 cr = __ldg(&S.sph[i].cr);
            const uint32_t m = __ldg(&S.sph[i].mat);
            fill_sphere(cr, m, o, d, t, rec);
            rec.sampled_light = S.sample_lights && (fbits(__ldg(&S.mat[m].ior_flags.y)) & PT_MF_EMITS) != 0;
            if (EXT && rec.sampled_light) {
                rec.lkind = 1;
                rec.lgeo = cr;
            }
            break;
        }
        case PT_HIT_TRIANGLE: {
            const float4* sl = S.slots + 3 * size_t(h.index);
            const uint32_t i = fbits(__ldg(sl + 2).y);
            rec.p = o + d * t;
            fill_triangle<TEX>(S, i, d, h.u, h.v, rec);
            // an emissive flat triangle of positive area is a light of the extended list
            if (EXT && S.sample_lights && (fbits(__ldg(&S.mat[rec.mat].ior_flags.y)) & PT_MF_EMITS)) {
                const float4 a = __ldg(sl), b = __ldg(sl + 1), c = __ldg(sl + 2);
                const float area = pt_triangle_area(a.w, b.x, b.y, b.z, b.w, c.x);
                if (area > 0.0f && area < 3.0e38f) {
                    const float4 fn = __ldg(&S.tri[i].fn);
                    rec.sampled_light = true;
                    rec.lkind = 2;
                    rec.lgeo = make_float4(fn.x, fn.y, fn.z, area);
                }
            }
            break;
        }
        case PT_HIT_INSTANCE: {
            const PtShadeInst* in = S.inst + h.inst;
            float4 rows[3] = {__ldg(&in->row[0]), __ldg(&in->row[1]), __ldg(&in->row[2])};
            const uint32_t tri_base = __ldg(&in->tri_base), over = __ldg(&in->material);
            const uint32_t sub = fbits(__ldg(S.slots + 3 * size_t(h.index) + 2).y);
            const V ld = aff_vector(rows, d);
            fill_triangle<TEX>(S, tri_base + sub, ld, h.u, h.v, rec);
            rec.p = o + d * t;
            rec.normal = normalize(aff_transposed(rows, rec.normal));
            if (over != PT_NONE) rec.mat = over;
            break;
        }
        default:
            break;
    }
}

// ---- random numbers (include/vec3.hpp:11-52) ------------------------------------------------
struct Rng {
    uint64_t s0, s1, s2, s3;
    // xoshiro256p::seed: splitmix64 across the four words.
    __device__ __forceinline__ void seed(uint64_t seed) {
        uint64_t* w[4] = {&s0, &s1, &s2, &s3};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint64_t z = (seed += 0x9e3779b97f4a7c15ull);
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            *w[k] = z ^ (z >> 31);
        }
    }
    __device__ __forceinline__ uint64_t next() {
        const uint64_t result = s0 + s3, t = s1 << 17;
        s2 ^= s0;
        s3 ^= s1;
        s1 ^= s2;
        s0 ^= s3;
        s2 ^= t;
        s3 = (s3 << 45) | (s3 >> 19);
        return result;
    }
    // random_real: the top 24 bits as a float in [0, 1).
    __device__ __forceinline__ float real() { return float(next() >> 40) * 0x1.0p-24f; }
};

// The per-(pixel, sample) stream of PT_RNG_SAMPLE: splitmix64's finaliser
// over (seed, row, column), then the sample number, seeds xoshiro256+.
__device__ __host__ __forceinline__ uint64_t sample_stream_seed(uint64_t seed, int i, int j, uint32_t s) {
    uint64_t x = seed ^ ((uint64_t(uint32_t(j)) << 32) | uint32_t(i));
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x ^ (uint64_t(s) * 0xd6e8feb86659fd93ull);
}

// ---- the Sobol sampler (include/sampler.hpp:35-127) -----------------------------------------
__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ uint32_t lk_permute(uint32_t x, uint32_t seed) {
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
// The second Sobol dimension, bit-reversed (sobol_1_reversed, sampler.hpp:91-94).
// Its direction numbers are Pascal's triangle mod 2, so bit m of the result
// is the parity of the set bits k of i with k a bitwise superset of m (Lucas'
// theorem): a superset-XOR transform over the 5-bit positions, five shift-and-
// mask steps instead of four table lookups.
__device__ __forceinline__ uint32_t sobol_1_reversed(uint32_t r) {
    r ^= (r >> 1) & 0x55555555u;
    r ^= (r >> 2) & 0x33333333u;
    r ^= (r >> 4) & 0x0f0f0f0fu;
    r ^= (r >> 8) & 0x00ff00ffu;
    r ^= (r >> 16) & 0x0000ffffu;
    return r;
}

struct Sampler {
    uint32_t pixel_seed, index;
    int base;
    // begin_sample (sampler.hpp:98-104)
    __device__ __forceinline__ void begin(uint64_t seed, int i, int j, uint32_t idx) {
        pixel_seed = hash_u32(uint32_t(i) * 0x9e3779b1u ^
                              hash_u32(uint32_t(j) ^ hash_u32(uint32_t(seed) ^ uint32_t(seed >> 32))));
        index = idx;
        base = 0;
    }
    // set_bounce (sampler.hpp:127)
    __device__ __forceinline__ void set_bounce(int k) { base = 1 + 2 * k; }
    // sample_2d (sampler.hpp:107-124): QMC for pairs 0..4, the random stream after.
    __device__ __forceinline__ void sample_2d(int pair_offset, Rng& rng, float& a, float& b) const {
        const int pair = base + pair_offset;
        if (pair > 4) {
            a = rng.real();
            b = rng.real();
            return;
        }
        const uint32_t seed = hash_u32(pixel_seed + uint32_t(pair) * 0x68bc21ebu);
        const uint32_t i = __brev(lk_permute(__brev(index), seed));
        const uint32_t x = __brev(lk_permute(i, seed ^ 0xa511e9b3u));
        const uint32_t y = __brev(lk_permute(sobol_1_reversed(i), seed ^ 0x63d83595u));
        a = float(x >> 8) * 0x1.0p-24f;
        b = float(y >> 8) * 0x1.0p-24f;
    }
};

// ---- materials (include/material.hpp) ----------------------------------------------------------
__device__ __forceinline__ V reflect(V v, V n) { return v - n * (2 * dot(v, n)); }
__device__ __forceinline__ V refract(V uv, V n, float ratio) {
    const float cos_theta = fminf(dot(-uv, n), 1.0f);
    const V r_perp = (uv + n * cos_theta) * ratio;
    const V r_parallel = n * -sqrtf(fabsf(1 - dot(r_perp, r_perp)));
    return r_perp + r_parallel;
}
// random_in_unit_sphere (vec3.hpp:121-127). vec3::random(-1, 1) builds the
// vector from three calls in one constructor argument list, which GCC on
// x86-64 evaluates right to left: z is drawn first, x last. The rejection
// loop is bounded: 64 misses in a row has probability 0.48^64 (~1e-20) for a
// real stream, but an all-zero xoshiro state (which a caller could supply
// as a snapshot) repeats (-1,-1,-1) forever; the bound turns that into a
// zero offset instead of a hung kernel.
__device__ __forceinline__ V random_in_unit_sphere(Rng& rng) {
    for (int tries = 0; tries < 64; ++tries) {
        const float z = -1.0f + 2.0f * rng.real();
        const float y = -1.0f + 2.0f * rng.real();
        const float x = -1.0f + 2.0f * rng.real();
        const V p = mk(x, y, z);
        if (dot(p, p) >= 1) continue;
        return p;
    }
    return mk(0, 0, 0);
}

// material::scatter for the four kinds: lambertian :59-74, metal :85-91,
// diffuse_light :97-102, dielectric :113-136.
__device__ __forceinline__ bool scatter(const PtMaterial& m, uint32_t type, V d_in, const Rec& rec,
                                        const Sampler& smp, Rng& rng, V& attenuation, V& dir) {
    if (type == PT_MAT_LAMBERTIAN) {
        float a, b;
        smp.sample_2d(0, rng, a, b);
        const float r = sqrtf(a), phi = 2 * float(M_PI) * b;
        const V n = rec.normal;
        const float sign = copysignf(1.0f, n.z);
        const float p = -1 / (sign + n.z), q = n.x * n.y * p;
        const V t1 = mk(1 + sign * n.x * n.x * p, sign * q, -sign * n.x);
        const V t2 = mk(q, sign + n.y * n.y * p, -n.y);
        float sp, cp;
        sin_cos(phi, sp, cp);
        dir = t1 * (r * cp) + t2 * (r * sp) + n * sqrtf(fmaxf(0.0f, 1 - a));
        attenuation = xyz(m.albedo_type);
        return true;
    }
    if (type == PT_MAT_METAL) {
        const V reflected = reflect(normalize(d_in), rec.normal);
        dir = reflected + random_in_unit_sphere(rng) * m.emission_fuzz.w;
        attenuation = xyz(m.albedo_type);
        return dot(dir, rec.normal) > 0;
    }
    if (type == PT_MAT_DIELECTRIC) {
        attenuation = mk(1, 1, 1);
        const float ior = m.ior_flags.x;
        const float ratio = rec.front_face ? (1 / ior) : ior;
        const V unit = normalize(d_in);
        const float cos_theta = fminf(dot(-unit, rec.normal), 1.0f);
        const float sin_theta = sqrtf(1 - cos_theta * cos_theta);
        const bool cannot_refract = ratio * sin_theta > 1;
        bool refl = cannot_refract;
        if (!refl) {
            // schlick (:131-136)
            float r0 = (1 - ratio) / (1 + ratio);
            r0 = r0 * r0;
            const float x = 1 - cos_theta, x2 = x * x;
            const float sch = r0 + (1 - r0) * x2 * x2 * x;
            refl = sch > rng.real();
        }
        dir = refl ? reflect(unit, rec.normal) : refract(unit, rec.normal, ratio);
        return true;
    }
    return false;  // diffuse_light
}

}  // namespace ptd
