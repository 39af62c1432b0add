// BVH build on the GPU, producing exactly the nodes and leaf order of the
// host builder (bvh_build.cpp) and so of the reference's bvh::build
// (include/bvh.hpp:39-52, split :126-197, collapse :205-242).
//
// The binary tree is built top-down:
//  * Nodes of more than kSmall primitives, level by level, with the work
//    spread over chunks of their primitive ranges: bounds and 16-bin
//    histograms by block reductions and atomics, the SAH sweep by one thread
//    per node, and the partition by ranks.
//  * Each node of at most kSmall primitives, with its whole subtree, by one
//    thread running the host builder's steps in the host builder's order.
// The 4-wide collapse then runs on the host over the downloaded binary tree.
//
// Exactness. The host builder grows boxes with std::min / std::max over the
// primitives in their current order; those keep the FIRST of equal values,
// which matters only for -0.0 against +0.0 but is still part of the output.
// The parallel reductions therefore order candidates by (value, position):
// a 64-bit key with the value's order-preserving bits above the position
// (its complement for maxima), both zeros mapped to one value, and the
// winning position's own float read back. std::partition (libstdc++, the
// bidirectional form) swaps the i-th primitive failing the predicate left of
// the split point with the i-th one passing it right of the split point,
// counted from the right; the rank kernels pair them the same way. All float
// arithmetic is the host builder's, in its order, without contraction.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/photon_cuda.h"
#include "pt_host.hpp"

namespace pt {
pt_status cuda_fail(cudaError_t e, const char* what);
}
using namespace pt;

namespace {

constexpr int kBins = 16;
constexpr uint32_t kMaxLeaf = 8;
constexpr int kMaxDepth = 64;
constexpr uint32_t kSmall = 128;  // subtrees at most this big: one thread each
constexpr uint32_t kChunk = 4096;  // primitive positions per block in the level kernels
constexpr int kThreads = 256;
constexpr int kItems = kChunk / kThreads;  // contiguous positions per thread
constexpr unsigned long long kEmptyMin = ~0ull, kEmptyMax = 0ull;

struct BNode {  // a node of the binary tree
    float mn[3], mx[3];
    uint32_t first, count;  // interior: first = left child (right = first + 1), count = 0
};

struct LNode {  // a node of the current level
    uint32_t bidx, first, count, depth;
};

struct Decision {
    int kind;  // 0 leaf, 1 SAH split (partition), 2 median split (no partition)
    int axis, cut;
    float lo, extent;
    uint32_t mid, n_swap;
};

struct Chunk {
    uint32_t node, begin, end;  // node: index into the level's arrays; [begin, end) positions
};

// std::min / std::max (the first of equal values is kept)
__host__ __device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__host__ __device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }

struct GBox {
    float mn[3], mx[3];
    __device__ void clear() {
        for (int a = 0; a < 3; ++a) {
            mn[a] = __int_as_float(0x7f800000);
            mx[a] = -__int_as_float(0x7f800000);
        }
    }
    __device__ void grow(const float* bmn, const float* bmx) {
        for (int a = 0; a < 3; ++a) {
            mn[a] = smin(mn[a], bmn[a]);
            mx[a] = smax(mx[a], bmx[a]);
        }
    }
    // aabb::half_area (include/aabb.hpp:26-30)
    __device__ float half_area() const {
        if (mn[0] > mx[0]) return 0;
        const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
        return dx * dy + dy * dz + dz * dx;
    }
};

__device__ __forceinline__ int bin_of(float c, float lo, float extent) {
    const int b = static_cast<int>(static_cast<float>(kBins) * (c - lo) / extent);
    return b < 0 ? 0 : b >= kBins ? kBins - 1 : b;
}

// Order-preserving bits of a float with -0.0 and +0.0 equal.
__device__ __forceinline__ uint32_t ord_bits(float f) {
    const uint32_t u = __float_as_uint(f);
    if ((u & 0x7fffffffu) == 0) return 0x80000000u;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ unsigned long long min_key(float v, uint32_t pos) {
    return (static_cast<unsigned long long>(ord_bits(v)) << 32) | pos;
}
__device__ __forceinline__ unsigned long long max_key(float v, uint32_t pos) {
    return (static_cast<unsigned long long>(ord_bits(v)) << 32) | (0xffffffffu - pos);
}

__device__ __forceinline__ unsigned long long warp_min(unsigned long long k) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, k, o);
        k = x < k ? x : k;
    }
    return k;
}
__device__ __forceinline__ unsigned long long warp_max(unsigned long long k) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, k, o);
        k = x > k ? x : k;
    }
    return k;
}

struct Prims {
    const float* box;     // 6 per primitive (min xyz, max xyz)
    const float* center;  // 3 per primitive
    uint32_t* order;
};

// The value a bound key names: coordinate c of the minimum (MAX = false) or
// maximum corner of the primitive at that position, or of its centroid.
__device__ float key_value(const Prims& P, unsigned long long key, bool is_max, bool centroid, int c) {
    if (key == (is_max ? kEmptyMax : kEmptyMin)) return is_max ? -__int_as_float(0x7f800000) : __int_as_float(0x7f800000);
    const uint32_t low = static_cast<uint32_t>(key & 0xffffffffu);
    const uint32_t pos = is_max ? 0xffffffffu - low : low;
    const uint32_t p = P.order[pos];
    if (centroid) return P.center[3 * size_t(p) + c];
    return P.box[6 * size_t(p) + (is_max ? 3 : 0) + c];
}

// ---- level kernels (nodes of more than kSmall primitives) -------------------------------
// Per node 12 keys: box min xyz, box max xyz, centroid min xyz, centroid max xyz.
__global__ void __launch_bounds__(kThreads) bounds_kernel(Prims P, const LNode* __restrict__ nodes,
                                                          const Chunk* __restrict__ chunks,
                                                          unsigned long long* __restrict__ keys) {
    __shared__ unsigned long long part[kThreads / 32][12];
    const Chunk ch = chunks[blockIdx.x];
    unsigned long long k[12];
    for (int q = 0; q < 12; ++q) k[q] = (q % 6) < 3 ? kEmptyMin : kEmptyMax;
    for (uint32_t pos = ch.begin + threadIdx.x; pos < ch.end; pos += kThreads) {
        const uint32_t p = P.order[pos];
        const float* b = P.box + 6 * size_t(p);
        const float* c = P.center + 3 * size_t(p);
        for (int a = 0; a < 3; ++a) {
            k[a] = min(k[a], min_key(b[a], pos));
            k[3 + a] = max(k[3 + a], max_key(b[3 + a], pos));
            k[6 + a] = min(k[6 + a], min_key(c[a], pos));
            k[9 + a] = max(k[9 + a], max_key(c[a], pos));
        }
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = 0; q < 12; ++q) {
        const unsigned long long r = (q % 6) < 3 ? warp_min(k[q]) : warp_max(k[q]);
        if (lane == 0) part[w][q] = r;
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        const int q = threadIdx.x;
        unsigned long long r = part[0][q];
        for (int i = 1; i < kThreads / 32; ++i) r = (q % 6) < 3 ? min(r, part[i][q]) : max(r, part[i][q]);
        if ((q % 6) < 3)
            atomicMin(keys + 12 * size_t(ch.node) + q, r);
        else
            atomicMax(keys + 12 * size_t(ch.node) + q, r);
    }
}

// Decodes each node's box and centroid bounds; writes the box into the binary tree.
__global__ void decode_kernel(Prims P, const LNode* __restrict__ nodes, uint32_t n, const unsigned long long* __restrict__ keys,
                              BNode* __restrict__ tree, float* __restrict__ cent) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long* k = keys + 12 * size_t(i);
    BNode& b = tree[nodes[i].bidx];
    for (int a = 0; a < 3; ++a) {
        b.mn[a] = key_value(P, k[a], false, false, a);
        b.mx[a] = key_value(P, k[3 + a], true, false, a);
        cent[6 * size_t(i) + a] = key_value(P, k[6 + a], false, true, a);
        cent[6 * size_t(i) + 3 + a] = key_value(P, k[9 + a], true, true, a);
    }
}

// Per node, axis and bin: 3 min keys, 3 max keys (the bin's box) and a count.
constexpr int kBinKeys = 3 * kBins * 6;
__global__ void __launch_bounds__(kThreads) bins_kernel(Prims P, const LNode* __restrict__ nodes,
                                                        const Chunk* __restrict__ chunks, const float* __restrict__ cent,
                                                        unsigned long long* __restrict__ bin_keys,
                                                        uint32_t* __restrict__ bin_count) {
    __shared__ unsigned long long sk[kBinKeys];
    __shared__ uint32_t sc[3 * kBins];
    const Chunk ch = chunks[blockIdx.x];
    const LNode nd = nodes[ch.node];
    if (nd.depth + 1 >= kMaxDepth) return;  // a leaf: no split is searched
    for (int i = threadIdx.x; i < kBinKeys; i += kThreads) sk[i] = ((i % 6) < 3) ? kEmptyMin : kEmptyMax;
    for (int i = threadIdx.x; i < 3 * kBins; i += kThreads) sc[i] = 0;
    __syncthreads();
    float lo[3], ext[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = cent[6 * size_t(ch.node) + a];
        ext[a] = cent[6 * size_t(ch.node) + 3 + a] - lo[a];
    }
    for (uint32_t pos = ch.begin + threadIdx.x; pos < ch.end; pos += kThreads) {
        const uint32_t p = P.order[pos];
        const float* b = P.box + 6 * size_t(p);
        const float* c = P.center + 3 * size_t(p);
        for (int axis = 0; axis < 3; ++axis) {
            if (!(ext[axis] > 0)) continue;
            const int bin = axis * kBins + bin_of(c[axis], lo[axis], ext[axis]);
            for (int a = 0; a < 3; ++a) {
                atomicMin(&sk[6 * bin + a], min_key(b[a], pos));
                atomicMax(&sk[6 * bin + 3 + a], max_key(b[3 + a], pos));
            }
            atomicAdd(&sc[bin], 1u);
        }
    }
    __syncthreads();
    unsigned long long* gk = bin_keys + size_t(kBinKeys) * ch.node;
    for (int i = threadIdx.x; i < kBinKeys; i += kThreads) {
        if ((i % 6) < 3) {
            if (sk[i] != kEmptyMin) atomicMin(gk + i, sk[i]);
        } else if (sk[i] != kEmptyMax) {
            atomicMax(gk + i, sk[i]);
        }
    }
    for (int i = threadIdx.x; i < 3 * kBins; i += kThreads)
        if (sc[i]) atomicAdd(bin_count + 3 * kBins * size_t(ch.node) + i, sc[i]);
}

// The split decision of split() (bvh.hpp:126-197), one thread per node.
__global__ void decide_kernel(Prims P, const LNode* __restrict__ nodes, uint32_t n, const BNode* __restrict__ tree,
                              const float* __restrict__ cent, const unsigned long long* __restrict__ bin_keys,
                              const uint32_t* __restrict__ bin_count, Decision* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const LNode nd = nodes[i];
    Decision d;
    d.kind = 0;
    d.axis = -1;
    d.cut = 0;
    d.lo = 0;
    d.extent = 0;
    d.mid = 0;
    d.n_swap = 0;
    if (nd.count == 1 || nd.depth + 1 >= kMaxDepth) {
        out[i] = d;
        return;
    }
    GBox box;
    const BNode& tb = tree[nd.bidx];
    for (int a = 0; a < 3; ++a) {
        box.mn[a] = tb.mn[a];
        box.mx[a] = tb.mx[a];
    }
    float best_cost = __int_as_float(0x7f800000);
    int best_axis = -1, best_bin = 0;
    const unsigned long long* K = bin_keys + size_t(kBinKeys) * i;
    const uint32_t* C = bin_count + 3 * kBins * size_t(i);
    for (int axis = 0; axis < 3; ++axis) {
        const float lo = cent[6 * size_t(i) + axis], extent = cent[6 * size_t(i) + 3 + axis] - lo;
        if (extent <= 0) continue;
        GBox bb[kBins];
        for (int b = 0; b < kBins; ++b) {
            const unsigned long long* k = K + 6 * (axis * kBins + b);
            for (int a = 0; a < 3; ++a) {
                bb[b].mn[a] = key_value(P, k[a], false, false, a);
                bb[b].mx[a] = key_value(P, k[3 + a], true, false, a);
            }
        }
        float right_area[kBins];
        uint32_t right_count[kBins];
        GBox acc;
        acc.clear();
        uint32_t cnt = 0;
        for (int b = kBins - 1; b > 0; --b) {
            acc.grow(bb[b].mn, bb[b].mx);
            cnt += C[axis * kBins + b];
            right_area[b] = acc.half_area();
            right_count[b] = cnt;
        }
        acc.clear();
        cnt = 0;
        for (int b = 0; b < kBins - 1; ++b) {
            acc.grow(bb[b].mn, bb[b].mx);
            cnt += C[axis * kBins + b];
            if (cnt == 0 || right_count[b + 1] == 0) continue;
            const float weighted = acc.half_area() * static_cast<float>(cnt) +
                                   right_area[b + 1] * static_cast<float>(right_count[b + 1]);
            const float cost = 1.0f + (1.0f * weighted) / box.half_area();
            if (cost < best_cost) {
                best_cost = cost;
                best_axis = axis;
                best_bin = b;
            }
        }
    }
    if (nd.count <= kMaxLeaf && !(best_cost < static_cast<float>(nd.count) * 1.0f)) {
        out[i] = d;
        return;
    }
    if (best_axis >= 0) {
        d.kind = 1;
        d.axis = best_axis;
        d.cut = best_bin;
        d.lo = cent[6 * size_t(i) + best_axis];
        d.extent = cent[6 * size_t(i) + 3 + best_axis] - d.lo;
        uint32_t left = 0;
        for (int b = 0; b <= best_bin; ++b) left += C[best_axis * kBins + b];
        d.mid = nd.first + left;
    } else {
        d.kind = 2;
        d.mid = nd.first + nd.count / 2;
    }
    out[i] = d;
}

__device__ __forceinline__ bool goes_left(const Prims& P, uint32_t p, const Decision& d) {
    return bin_of(P.center[3 * size_t(p) + d.axis], d.lo, d.extent) <= d.cut;
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ uint32_t block_scan(uint32_t v, uint32_t& excl) {
    __shared__ uint32_t warp_tot[kThreads / 32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int i = 0; i < kThreads / 32; ++i) {
        if (i < w) before += warp_tot[i];
        total += warp_tot[i];
    }
    __syncthreads();
    excl = before + x - v;
    return total;
}

// Per chunk of an SAH-split node: how many primitives left of the split
// point fail the predicate ("L") and right of it pass it ("R").
__global__ void __launch_bounds__(kThreads) part_count_kernel(Prims P, const Chunk* __restrict__ chunks,
                                                              const Decision* __restrict__ dec,
                                                              uint32_t* __restrict__ cl, uint32_t* __restrict__ cr) {
    const Chunk ch = chunks[blockIdx.x];
    const Decision d = dec[ch.node];
    if (d.kind != 1) return;
    uint32_t nl = 0, nr = 0;
    for (uint32_t pos = ch.begin + threadIdx.x; pos < ch.end; pos += kThreads) {
        const bool left = goes_left(P, P.order[pos], d);
        nl += (pos < d.mid && !left) ? 1u : 0u;
        nr += (pos >= d.mid && left) ? 1u : 0u;
    }
    uint32_t e;
    const uint32_t tl = block_scan(nl, e);
    const uint32_t tr = block_scan(nr, e);
    if (threadIdx.x == 0) {
        cl[blockIdx.x] = tl;
        cr[blockIdx.x] = tr;
    }
}

// Per node, over its chunks (consecutive): L offsets from the left, R
// offsets from the right, and the number of swaps.
__global__ void part_scan_kernel(const LNode* __restrict__ nodes, uint32_t n, const uint32_t* __restrict__ chunk_begin,
                                 const uint32_t* __restrict__ chunk_end, uint32_t* __restrict__ cl,
                                 uint32_t* __restrict__ cr, Decision* __restrict__ dec, int* __restrict__ error) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || dec[i].kind != 1) return;
    uint32_t s = 0;
    for (uint32_t c = chunk_begin[i]; c < chunk_end[i]; ++c) {
        const uint32_t v = cl[c];
        cl[c] = s;
        s += v;
    }
    uint32_t r = 0;
    for (uint32_t c = chunk_end[i]; c-- > chunk_begin[i];) {
        const uint32_t v = cr[c];
        cr[c] = r;
        r += v;
    }
    dec[i].n_swap = s;
    if (s != r) {  // the bin counts and the predicate disagree: never expected
        atomicExch(error, 3);
        dec[i].n_swap = 0;
    }
}

// The positions of the i-th L (from the left) and the i-th R (from the right).
__global__ void __launch_bounds__(kThreads) part_rank_kernel(Prims P, const LNode* __restrict__ nodes,
                                                             const Chunk* __restrict__ chunks,
                                                             const Decision* __restrict__ dec,
                                                             const uint32_t* __restrict__ cl,
                                                             const uint32_t* __restrict__ cr,
                                                             uint32_t* __restrict__ lpos, uint32_t* __restrict__ rpos) {
    const Chunk ch = chunks[blockIdx.x];
    const Decision d = dec[ch.node];
    if (d.kind != 1) return;
    const uint32_t base = nodes[ch.node].first;
    // this thread's contiguous positions
    const uint32_t b0 = ch.begin + threadIdx.x * kItems;
    uint32_t flags = 0;  // bit j: L at b0 + j; bit 16 + j: R at b0 + j
    for (int j = 0; j < kItems; ++j) {
        const uint32_t pos = b0 + j;
        if (pos >= ch.end) break;
        const bool left = goes_left(P, P.order[pos], d);
        if (pos < d.mid && !left) flags |= 1u << j;
        if (pos >= d.mid && left) flags |= 1u << (16 + j);
    }
    const uint32_t nl = __popc(flags & 0xffffu), nr = __popc(flags >> 16);
    uint32_t el, er;
    block_scan(nl, el);
    const uint32_t tr = block_scan(nr, er);
    uint32_t li = cl[blockIdx.x] + el;
    // R ranks count from the right: those after this position in the chunk, plus later chunks
    uint32_t rafter = cr[blockIdx.x] + (tr - er - nr);
    for (int j = kItems - 1; j >= 0; --j) {
        if (flags & (1u << (16 + j))) rpos[base + rafter++] = b0 + j;
    }
    for (int j = 0; j < kItems; ++j)
        if (flags & (1u << j)) lpos[base + li++] = b0 + j;
}

__global__ void part_swap_kernel(Prims P, const LNode* __restrict__ nodes, const Chunk* __restrict__ chunks,
                                 const Decision* __restrict__ dec, const uint32_t* __restrict__ lpos,
                                 const uint32_t* __restrict__ rpos, int* __restrict__ error) {
    const Chunk ch = chunks[blockIdx.x];
    const Decision d = dec[ch.node];
    if (d.kind != 1) return;
    const uint32_t first = nodes[ch.node].first, end = first + nodes[ch.node].count;
    for (uint32_t pos = ch.begin + threadIdx.x; pos < ch.end; pos += kThreads) {
        const uint32_t i = pos - first;
        if (i >= d.n_swap) continue;
        const uint32_t a = lpos[first + i], b = rpos[first + i];
        if (a < first || a >= d.mid || b < d.mid || b >= end) {  // never expected: not a valid pair
            atomicExch(error, 4);
            continue;
        }
        const uint32_t t = P.order[a];
        P.order[a] = P.order[b];
        P.order[b] = t;
    }
}

// ---- small subtrees: one thread each, the host builder's steps ------------------------------
__global__ void small_kernel(Prims P, const LNode* __restrict__ roots, uint32_t n_roots, BNode* __restrict__ tree,
                             uint32_t* __restrict__ next_node, uint32_t capacity, int* __restrict__ error) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_roots) return;
    uint32_t stack_idx[kMaxDepth + 2], stack_depth[kMaxDepth + 2];
    int top = 0;
    stack_idx[top] = roots[r].bidx;
    stack_depth[top++] = roots[r].depth;
    while (top > 0) {
        --top;
        const uint32_t idx = stack_idx[top], depth = stack_depth[top];
        BNode& node = tree[idx];
        const uint32_t first = node.first, count = node.count;
        GBox box, cb;
        box.clear();
        cb.clear();
        for (uint32_t i = first; i < first + count; ++i) {
            const uint32_t p = P.order[i];
            box.grow(P.box + 6 * size_t(p), P.box + 6 * size_t(p) + 3);
            cb.grow(P.center + 3 * size_t(p), P.center + 3 * size_t(p));
        }
        for (int a = 0; a < 3; ++a) {
            node.mn[a] = box.mn[a];
            node.mx[a] = box.mx[a];
        }
        if (count == 1 || depth + 1 >= kMaxDepth) continue;
        float best_cost = __int_as_float(0x7f800000);
        int best_axis = -1, best_bin = 0;
        for (int axis = 0; axis < 3; ++axis) {
            const float lo = cb.mn[axis], extent = cb.mx[axis] - lo;
            if (extent <= 0) continue;
            GBox bb[kBins];
            uint32_t bc[kBins];
            for (int b = 0; b < kBins; ++b) {
                bb[b].clear();
                bc[b] = 0;
            }
            for (uint32_t i = first; i < first + count; ++i) {
                const uint32_t p = P.order[i];
                const int b = bin_of(P.center[3 * size_t(p) + axis], lo, extent);
                bb[b].grow(P.box + 6 * size_t(p), P.box + 6 * size_t(p) + 3);
                ++bc[b];
            }
            float right_area[kBins];
            uint32_t right_count[kBins];
            GBox acc;
            acc.clear();
            uint32_t cnt = 0;
            for (int b = kBins - 1; b > 0; --b) {
                acc.grow(bb[b].mn, bb[b].mx);
                cnt += bc[b];
                right_area[b] = acc.half_area();
                right_count[b] = cnt;
            }
            acc.clear();
            cnt = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                acc.grow(bb[b].mn, bb[b].mx);
                cnt += bc[b];
                if (cnt == 0 || right_count[b + 1] == 0) continue;
                const float weighted = acc.half_area() * static_cast<float>(cnt) +
                                       right_area[b + 1] * static_cast<float>(right_count[b + 1]);
                const float cost = 1.0f + (1.0f * weighted) / box.half_area();
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = axis;
                    best_bin = b;
                }
            }
        }
        if (count <= kMaxLeaf && !(best_cost < static_cast<float>(count) * 1.0f)) continue;
        uint32_t mid;
        if (best_axis >= 0) {
            // std::partition, bidirectional form
            const float lo = cb.mn[best_axis], extent = cb.mx[best_axis] - lo;
            uint32_t a = first, e = first + count;
            while (true) {
                while (a != e && bin_of(P.center[3 * size_t(P.order[a]) + best_axis], lo, extent) <= best_bin) ++a;
                if (a == e) break;
                --e;
                while (a != e && !(bin_of(P.center[3 * size_t(P.order[e]) + best_axis], lo, extent) <= best_bin)) --e;
                if (a == e) break;
                const uint32_t t = P.order[a];
                P.order[a] = P.order[e];
                P.order[e] = t;
                ++a;
            }
            mid = a;
        } else {
            mid = first + count / 2;
        }
        const uint32_t left = atomicAdd(next_node, 2u);
        if (left + 2 > capacity) {
            atomicExch(error, 1);
            return;
        }
        tree[left].first = first;
        tree[left].count = mid - first;
        tree[left + 1].first = mid;
        tree[left + 1].count = first + count - mid;
        node.first = left;
        node.count = 0;
        if (top + 2 > kMaxDepth + 2) {
            atomicExch(error, 2);
            return;
        }
        stack_idx[top] = left + 1;
        stack_depth[top++] = depth + 1;
        stack_idx[top] = left;
        stack_depth[top++] = depth + 1;
    }
}

// Empty keys: minima all ones, maxima zero (q % 6 < 3 are minima in both key arrays).
__global__ void init_keys_kernel(unsigned long long* __restrict__ keys, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        keys[i] = (i % 6) < 3 ? kEmptyMin : kEmptyMax;
}

struct TreeUpdate {
    uint32_t idx, first, count;
};

// Sets first / count of binary nodes (new children, and parents that become interior).
__global__ void update_kernel(BNode* __restrict__ tree, const TreeUpdate* __restrict__ u, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    tree[u[i].idx].first = u[i].first;
    tree[u[i].idx].count = u[i].count;
}

__global__ void prepare_kernel(const float* __restrict__ boxes, uint32_t n, float* __restrict__ center,
                               uint32_t* __restrict__ order) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int a = 0; a < 3; ++a) center[3 * size_t(i) + a] = (boxes[6 * size_t(i) + a] + boxes[6 * size_t(i) + 3 + a]) * 0.5f;
        order[i] = i;
    }
}

template <class T>
struct DevArray {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t want) {
        if (want <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        const cudaError_t e = cudaMalloc(&p, std::max<size_t>(want, 1) * sizeof(T));
        if (!e) n = want;
        return e;
    }
    ~DevArray() {
        if (p) cudaFree(p);
    }
};

cudaError_t build_device(const float* h_boxes, uint32_t n, std::vector<float>& boxes_out, std::vector<uint32_t>& first,
                         std::vector<uint32_t>& count, std::vector<uint32_t>& order, int& device_error) {
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e) return e;
    const uint32_t capacity = 2 * n;
    DevArray<float> d_box, d_center, d_cent;
    DevArray<uint32_t> d_order, d_lpos, d_rpos, d_next, d_bin_count, d_cl, d_cr, d_cb, d_ce;
    DevArray<BNode> d_tree;
    DevArray<LNode> d_nodes, d_small;
    DevArray<Chunk> d_chunks;
    DevArray<unsigned long long> d_keys, d_bin_keys;
    DevArray<Decision> d_dec;
    DevArray<int> d_err;
    if (!e) e = d_box.ensure(6 * size_t(n));
    if (!e) e = d_center.ensure(3 * size_t(n));
    if (!e) e = d_order.ensure(n);
    if (!e) e = d_lpos.ensure(n);
    if (!e) e = d_rpos.ensure(n);
    if (!e) e = d_tree.ensure(capacity);
    if (!e) e = d_next.ensure(1);
    if (!e) e = d_err.ensure(1);
    if (!e) e = cudaMemcpyAsync(d_box.p, h_boxes, 6 * size_t(n) * sizeof(float), cudaMemcpyHostToDevice, st);
    if (!e) e = cudaMemsetAsync(d_err.p, 0, sizeof(int), st);
    if (!e) {
        prepare_kernel<<<std::min<uint32_t>((n + 255) / 256, 148 * 8), 256, 0, st>>>(d_box.p, n, d_center.p, d_order.p);
        e = cudaGetLastError();
    }
    const Prims P{d_box.p, d_center.p, d_order.p};

    // The binary tree's node records live on the device; the host knows the
    // large nodes' children, which it allocates.
    uint32_t n_tree = 1;
    BNode root{};
    root.first = 0;
    root.count = n;
    if (!e) e = cudaMemcpyAsync(d_tree.p, &root, sizeof(BNode), cudaMemcpyHostToDevice, st);
    std::vector<LNode> level, small;
    if (n > kSmall)
        level.push_back({0, 0, n, 0});
    else
        small.push_back({0, 0, n, 0});
    std::vector<Chunk> chunks;
    std::vector<uint32_t> cbeg, cend;
    std::vector<Decision> dec;
    std::vector<TreeUpdate> updates;
    DevArray<TreeUpdate> d_updates;
    while (!e && !level.empty()) {
        const uint32_t L = uint32_t(level.size());
        chunks.clear();
        cbeg.resize(L);
        cend.resize(L);
        for (uint32_t i = 0; i < L; ++i) {
            cbeg[i] = uint32_t(chunks.size());
            for (uint32_t b = level[i].first; b < level[i].first + level[i].count; b += kChunk)
                chunks.push_back({i, b, std::min(b + kChunk, level[i].first + level[i].count)});
            cend[i] = uint32_t(chunks.size());
        }
        const uint32_t C = uint32_t(chunks.size());
        if (!e) e = d_nodes.ensure(L);
        if (!e) e = d_chunks.ensure(C);
        if (!e) e = d_keys.ensure(12 * size_t(L));
        if (!e) e = d_cent.ensure(6 * size_t(L));
        if (!e) e = d_bin_keys.ensure(size_t(kBinKeys) * L);
        if (!e) e = d_bin_count.ensure(3 * kBins * size_t(L));
        if (!e) e = d_dec.ensure(L);
        if (!e) e = d_cl.ensure(C);
        if (!e) e = d_cr.ensure(C);
        if (!e) e = d_cb.ensure(L);
        if (!e) e = d_ce.ensure(L);
        if (e) break;
        e = cudaMemcpyAsync(d_nodes.p, level.data(), L * sizeof(LNode), cudaMemcpyHostToDevice, st);
        if (!e) e = cudaMemcpyAsync(d_chunks.p, chunks.data(), C * sizeof(Chunk), cudaMemcpyHostToDevice, st);
        if (!e) {
            init_keys_kernel<<<std::min<size_t>((12 * size_t(L) + 255) / 256, 1184), 256, 0, st>>>(d_keys.p, 12 * size_t(L));
            init_keys_kernel<<<std::min<size_t>((size_t(kBinKeys) * L + 255) / 256, 1184), 256, 0, st>>>(
                d_bin_keys.p, size_t(kBinKeys) * L);
            e = cudaGetLastError();
        }
        if (!e) e = cudaMemsetAsync(d_bin_count.p, 0, 3 * kBins * size_t(L) * 4, st);
        if (!e) e = cudaMemcpyAsync(d_cb.p, cbeg.data(), L * 4, cudaMemcpyHostToDevice, st);
        if (!e) e = cudaMemcpyAsync(d_ce.p, cend.data(), L * 4, cudaMemcpyHostToDevice, st);
        if (e) break;
        bounds_kernel<<<C, kThreads, 0, st>>>(P, d_nodes.p, d_chunks.p, d_keys.p);
        decode_kernel<<<(L + 127) / 128, 128, 0, st>>>(P, d_nodes.p, L, d_keys.p, d_tree.p, d_cent.p);
        bins_kernel<<<C, kThreads, 0, st>>>(P, d_nodes.p, d_chunks.p, d_cent.p, d_bin_keys.p, d_bin_count.p);
        decide_kernel<<<(L + 63) / 64, 64, 0, st>>>(P, d_nodes.p, L, d_tree.p, d_cent.p, d_bin_keys.p, d_bin_count.p,
                                                    d_dec.p);
        part_count_kernel<<<C, kThreads, 0, st>>>(P, d_chunks.p, d_dec.p, d_cl.p, d_cr.p);
        part_scan_kernel<<<(L + 127) / 128, 128, 0, st>>>(d_nodes.p, L, d_cb.p, d_ce.p, d_cl.p, d_cr.p, d_dec.p, d_err.p);
        part_rank_kernel<<<C, kThreads, 0, st>>>(P, d_nodes.p, d_chunks.p, d_dec.p, d_cl.p, d_cr.p, d_lpos.p, d_rpos.p);
        part_swap_kernel<<<C, kThreads, 0, st>>>(P, d_nodes.p, d_chunks.p, d_dec.p, d_lpos.p, d_rpos.p, d_err.p);
        e = cudaGetLastError();
        dec.resize(L);
        if (!e) e = cudaMemcpyAsync(dec.data(), d_dec.p, L * sizeof(Decision), cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (e) break;
        // Children of the split nodes: records for the device tree, and the next level.
        std::vector<LNode> next;
        updates.clear();
        for (uint32_t i = 0; i < L; ++i) {
            const LNode& nd = level[i];
            if (dec[i].kind == 0) continue;  // a leaf: its record (first, count) is already right
            const uint32_t left = n_tree;
            n_tree += 2;
            const uint32_t mid = dec[i].mid;
            const LNode kids[2] = {{left, nd.first, mid - nd.first, nd.depth + 1},
                                   {left + 1, mid, nd.first + nd.count - mid, nd.depth + 1}};
            for (int c = 0; c < 2; ++c) {
                updates.push_back({kids[c].bidx, kids[c].first, kids[c].count});
                (kids[c].count > kSmall ? next : small).push_back(kids[c]);
            }
            updates.push_back({nd.bidx, left, 0u});  // the parent becomes interior; its box stays
        }
        if (!updates.empty()) {
            const uint32_t U = uint32_t(updates.size());
            e = d_updates.ensure(U);
            if (!e) e = cudaMemcpyAsync(d_updates.p, updates.data(), U * sizeof(TreeUpdate), cudaMemcpyHostToDevice, st);
            if (!e) {
                update_kernel<<<(U + 255) / 256, 256, 0, st>>>(d_tree.p, d_updates.p, U);
                e = cudaGetLastError();
            }
            // the host vector must outlive its copy
            if (!e) e = cudaStreamSynchronize(st);
        }
        level.swap(next);
    }
    if (!e && !small.empty()) {
        if (!e) e = d_small.ensure(small.size());
        if (!e) e = cudaMemcpyAsync(d_small.p, small.data(), small.size() * sizeof(LNode), cudaMemcpyHostToDevice, st);
        if (!e) e = cudaMemcpyAsync(d_next.p, &n_tree, 4, cudaMemcpyHostToDevice, st);
        if (!e) {
            const uint32_t ns = uint32_t(small.size());
            small_kernel<<<(ns + 63) / 64, 64, 0, st>>>(P, d_small.p, ns, d_tree.p, d_next.p, capacity, d_err.p);
            e = cudaGetLastError();
        }
        if (!e) e = cudaMemcpyAsync(&n_tree, d_next.p, 4, cudaMemcpyDeviceToHost, st);
    }
    if (!e) e = cudaMemcpyAsync(&device_error, d_err.p, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    std::vector<BNode> tree;
    if (!e && !device_error) {
        n_tree = std::min(n_tree, capacity);
        tree.resize(n_tree);
        order.resize(n);
        e = cudaMemcpyAsync(tree.data(), d_tree.p, n_tree * sizeof(BNode), cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaMemcpyAsync(order.data(), d_order.p, size_t(n) * 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
    }
    cudaStreamDestroy(st);
    if (e || device_error) return e;
    boxes_out.resize(6 * size_t(n_tree));
    first.resize(n_tree);
    count.resize(n_tree);
    for (uint32_t i = 0; i < n_tree; ++i) {
        for (int a = 0; a < 3; ++a) {
            boxes_out[6 * size_t(i) + a] = tree[i].mn[a];
            boxes_out[6 * size_t(i) + 3 + a] = tree[i].mx[a];
        }
        first[i] = tree[i].first;
        count[i] = tree[i].count;
    }
    return cudaSuccess;
}

}  // namespace

extern "C" pt_status pt_bvh_build_gpu(const float* boxes, uint32_t n, pt_bvh_node** nodes, uint32_t* n_nodes,
                                      uint32_t** order) {
    clear_error();
    if (!nodes || !n_nodes || !order || (n && !boxes)) return fail(PT_ERR_INVALID_ARG, "pt_bvh_build_gpu: null pointer");
    if (n > (1u << 30)) return fail(PT_ERR_INVALID_ARG, "pt_bvh_build_gpu: more than 2^30 primitives");
    *nodes = nullptr;
    *order = nullptr;
    *n_nodes = 0;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PT_ERR_NO_DEVICE, "no CUDA device");
    std::vector<pt_bvh_node> out;
    std::vector<uint32_t> ord;
    if (n > 0) {
        std::vector<float> bboxes;
        std::vector<uint32_t> bfirst, bcount;
        int derr = 0;
        if (cudaError_t e = build_device(boxes, n, bboxes, bfirst, bcount, ord, derr)) return cuda_fail(e, "pt_bvh_build_gpu");
        if (derr) return fail(PT_ERR_CUDA, "pt_bvh_build_gpu: internal consistency check failed (" + std::to_string(derr) + ")");
        collapse_bvh(bboxes.data(), bfirst.data(), bcount.data(), uint32_t(bfirst.size()), out);
    }
    pt_bvh_node* nb = static_cast<pt_bvh_node*>(std::malloc(std::max<size_t>(out.size(), 1) * sizeof(pt_bvh_node)));
    uint32_t* ob = static_cast<uint32_t*>(std::malloc(std::max<size_t>(ord.size(), 1) * sizeof(uint32_t)));
    if (!nb || !ob) {
        std::free(nb);
        std::free(ob);
        return fail(PT_ERR_OUT_OF_MEMORY, "pt_bvh_build_gpu: out of host memory");
    }
    if (!out.empty()) std::memcpy(nb, out.data(), out.size() * sizeof(pt_bvh_node));
    if (!ord.empty()) std::memcpy(ob, ord.data(), ord.size() * sizeof(uint32_t));
    *nodes = nb;
    *n_nodes = uint32_t(out.size());
    *order = ob;
    return PT_OK;
}
