// Host BVH builder. It must produce exactly the nodes and leaf order of the
// reference's bvh::build (include/bvh.hpp:39-52, split :126-197, collapse
// :205-242, bin_of :244-247), because closest-hit results are compared
// bit for bit and ties between equal-t primitives are decided by the order
// leaves are visited in. So the steps are the same: a binary tree by binned
// SAH (16 bins on the centroid extent, costs 1 + area-weighted counts over
// the parent's half area, a leaf kept when it holds <= 8 primitives and no
// split is cheaper than testing them, depth limit 64, std::partition on the
// chosen bin), then a collapse into 4-wide nodes that repeatedly opens the
// interior child with the largest half area. Float arithmetic is kept in the
// same order (compiled with -ffp-contract=off).
#include "pt_host.hpp"

#include <algorithm>
#include <limits>
#include <vector>

namespace pt {

namespace {

struct Box {
    float mn[3], mx[3];
    Box() {
        const float inf = std::numeric_limits<float>::infinity();
        for (int a = 0; a < 3; ++a) { mn[a] = inf; mx[a] = -inf; }
    }
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::min(mn[a], b.mn[a]);
            mx[a] = std::max(mx[a], b.mx[a]);
        }
    }
    void grow_point(const float p[3]) {
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::min(mn[a], p[a]);
            mx[a] = std::max(mx[a], p[a]);
        }
    }
    // aabb::half_area (include/aabb.hpp:26-30)
    float half_area() const {
        if (mn[0] > mx[0]) return 0;
        const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
        return dx * dy + dy * dz + dz * dx;
    }
};

struct BinNode {
    Box box;
    uint32_t first;  // interior: left child index (right = first + 1); leaf: start in order
    uint32_t count;  // 0 for interior
};

constexpr int kMaxDepth = 64;
constexpr int kBins = 16;
constexpr uint32_t kMaxLeaf = 8;

// The 4-wide collapse (include/bvh.hpp:205-242): from the binary root, open
// the interior child with the largest half area until four children, then
// recurse into interior children, numbering nodes in that (preorder) order.
uint32_t collapse_node(const std::vector<BinNode>& bin, uint32_t b, std::vector<pt_bvh_node>& nodes) {
    uint32_t child[4] = {b, 0, 0, 0};
    int n = 1;
    while (n < 4) {
        int widest = -1;
        float widest_area = -1;
        for (int i = 0; i < n; ++i) {
            const BinNode& c = bin[child[i]];
            if (c.count == 0 && c.box.half_area() > widest_area) {
                widest = i;
                widest_area = c.box.half_area();
            }
        }
        if (widest < 0) break;
        const uint32_t left = bin[child[widest]].first;
        child[widest] = left;
        child[n++] = left + 1;
    }
    const uint32_t index = static_cast<uint32_t>(nodes.size());
    nodes.emplace_back();
    pt_bvh_node nd;
    const float inf = std::numeric_limits<float>::infinity();
    for (int i = 0; i < 4; ++i) {
        for (int a = 0; a < 3; ++a) {
            nd.lo[a][i] = i < n ? bin[child[i]].box.mn[a] : inf;
            nd.hi[a][i] = i < n ? bin[child[i]].box.mx[a] : inf;
        }
        nd.first[i] = 0;
        nd.count[i] = 0;
        if (i >= n) continue;
        if (bin[child[i]].count > 0) {
            nd.first[i] = bin[child[i]].first;
            nd.count[i] = bin[child[i]].count;
        } else {
            nd.first[i] = collapse_node(bin, child[i], nodes);
        }
    }
    nodes[index] = nd;
    return index;
}

void collapse_binary(const std::vector<BinNode>& bin, std::vector<pt_bvh_node>& nodes) {
    nodes.clear();
    if (!bin.empty()) collapse_node(bin, 0, nodes);
}

class Builder {
public:
    Builder(const float* boxes, uint32_t n) : n_(n) {
        prims_.resize(n);
        centers_.resize(3 * size_t(n));
        for (uint32_t i = 0; i < n; ++i) {
            Box& b = prims_[i];
            for (int a = 0; a < 3; ++a) {
                b.mn[a] = boxes[6 * size_t(i) + a];
                b.mx[a] = boxes[6 * size_t(i) + 3 + a];
            }
            // aabb::center: (min + max) * 0.5
            for (int a = 0; a < 3; ++a) centers_[3 * size_t(i) + a] = (b.mn[a] + b.mx[a]) * 0.5f;
        }
    }

    void run(std::vector<pt_bvh_node>& nodes, std::vector<uint32_t>& order) {
        nodes.clear();
        order.resize(n_);
        for (uint32_t i = 0; i < n_; ++i) order[i] = i;
        if (n_ == 0) return;
        order_ = &order;
        bin_.reserve(2 * size_t(n_));
        bin_.push_back({Box(), 0, n_});
        split(0, 0);
        collapse_binary(bin_, nodes);
    }

private:
    static int bin_of(float c, float lo, float extent) {
        int b = static_cast<int>(kBins * (c - lo) / extent);
        return b < 0 ? 0 : b >= kBins ? kBins - 1 : b;
    }

    void split(uint32_t index, int depth) {
        std::vector<uint32_t>& order = *order_;
        const uint32_t first = bin_[index].first, count = bin_[index].count;
        Box box, centroids;
        for (uint32_t i = first; i < first + count; ++i) {
            box.grow(prims_[order[i]]);
            centroids.grow_point(&centers_[3 * size_t(order[i])]);
        }
        bin_[index].box = box;
        if (count == 1 || depth + 1 >= kMaxDepth) return;

        float best_cost = std::numeric_limits<float>::infinity();
        int best_axis = -1, best_bin = 0;
        for (int axis = 0; axis < 3; ++axis) {
            const float lo = centroids.mn[axis], extent = centroids.mx[axis] - lo;
            if (extent <= 0) continue;
            Box bin_box[kBins];
            uint32_t bin_count[kBins] = {};
            for (uint32_t i = first; i < first + count; ++i) {
                const int b = bin_of(centers_[3 * size_t(order[i]) + axis], lo, extent);
                bin_box[b].grow(prims_[order[i]]);
                ++bin_count[b];
            }
            float right_area[kBins];
            uint32_t right_count[kBins];
            Box acc;
            uint32_t n = 0;
            for (int b = kBins - 1; b > 0; --b) {
                acc.grow(bin_box[b]);
                n += bin_count[b];
                right_area[b] = acc.half_area();
                right_count[b] = n;
            }
            acc = Box();
            n = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                acc.grow(bin_box[b]);
                n += bin_count[b];
                if (n == 0 || right_count[b + 1] == 0) continue;
                // 1 + 1 * (A_l * n_l + A_r * n_r) / A_parent, in this order
                const float weighted = acc.half_area() * static_cast<float>(n) +
                                       right_area[b + 1] * static_cast<float>(right_count[b + 1]);
                const float cost = 1.0f + (1.0f * weighted) / box.half_area();
                if (cost < best_cost) { best_cost = cost; best_axis = axis; best_bin = b; }
            }
        }

        if (count <= kMaxLeaf && !(best_cost < static_cast<float>(count) * 1.0f)) return;

        uint32_t mid;
        if (best_axis >= 0) {
            const float lo = centroids.mn[best_axis], extent = centroids.mx[best_axis] - lo;
            const float* centers = centers_.data();
            const int axis = best_axis, cut = best_bin;
            uint32_t* m = std::partition(order.data() + first, order.data() + first + count, [&](uint32_t p) {
                return bin_of(centers[3 * size_t(p) + axis], lo, extent) <= cut;
            });
            mid = static_cast<uint32_t>(m - order.data());
        } else {
            mid = first + count / 2;
        }

        const uint32_t left = static_cast<uint32_t>(bin_.size());
        bin_.push_back({Box(), first, mid - first});
        bin_.push_back({Box(), mid, first + count - mid});
        bin_[index].first = left;
        bin_[index].count = 0;
        split(left, depth + 1);
        split(left + 1, depth + 1);
    }

    uint32_t n_;
    std::vector<Box> prims_;
    std::vector<float> centers_;
    std::vector<BinNode> bin_;
    std::vector<uint32_t>* order_ = nullptr;
};

}  // namespace

void collapse_bvh(const float* boxes, const uint32_t* first, const uint32_t* count, uint32_t n_bin,
                  std::vector<pt_bvh_node>& nodes) {
    std::vector<BinNode> bin(n_bin);
    for (uint32_t i = 0; i < n_bin; ++i) {
        for (int a = 0; a < 3; ++a) {
            bin[i].box.mn[a] = boxes[6 * size_t(i) + a];
            bin[i].box.mx[a] = boxes[6 * size_t(i) + 3 + a];
        }
        bin[i].first = first[i];
        bin[i].count = count[i];
    }
    collapse_binary(bin, nodes);
}

void build_bvh(const float* boxes, uint32_t n, std::vector<pt_bvh_node>& nodes, std::vector<uint32_t>& order) {
    Builder b(boxes, n);
    b.run(nodes, order);
}

// triangle::bounding_box (include/triangle.hpp:76-83): min/max of the three
// corners as given (p0, p1, p2 -- not p0 + e1, which can be an ulp off),
// padded by 1e-4.
void triangle_box(const float p0[3], const float p1[3], const float p2[3], float out[6]) {
    const float pad = 1e-4f;
    for (int a = 0; a < 3; ++a) {
        out[a] = std::min({p0[a], p1[a], p2[a]}) - pad;
        out[3 + a] = std::max({p0[a], p1[a], p2[a]}) + pad;
    }
}

// sphere::bounding_box (include/sphere.hpp:60-64)
void sphere_box(const float c[3], float r, float out[6]) {
    const float ar = std::fabs(r);
    for (int a = 0; a < 3; ++a) {
        out[a] = c[a] - ar;
        out[3 + a] = c[a] + ar;
    }
}

// affine::box (include/transform.hpp:62-70): the box around the 8 moved corners.
void affine_box(const pt_affine& x, const float in[6], float out[6]) {
    Box acc;
    for (int k = 0; k < 8; ++k) {
        const float c[3] = {k & 1 ? in[3] : in[0], k & 2 ? in[4] : in[1], k & 4 ? in[5] : in[2]};
        float p[3];
        affine_point(x, c, p);
        acc.grow_point(p);
    }
    for (int a = 0; a < 3; ++a) {
        out[a] = acc.mn[a];
        out[3 + a] = acc.mx[a];
    }
}

void affine_vector(const pt_affine& x, const float v[3], float out[3]) {
    for (int r = 0; r < 3; ++r) out[r] = x.m[r][0] * v[0] + x.m[r][1] * v[1] + x.m[r][2] * v[2];
}

void affine_point(const pt_affine& x, const float p[3], float out[3]) {
    float v[3];
    affine_vector(x, p, v);
    for (int r = 0; r < 3; ++r) out[r] = v[r] + x.t[r];
}

// affine::inverse (include/transform.hpp:42-59): cofactors in double, then
// t = -(M^-1 t) in float.
pt_affine affine_inverse(const pt_affine& x) {
    double a[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[i][j] = x.m[i][j];
    const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    const double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    const double inv[3][3] = {
        {c00 / det, (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det, (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det},
        {c01 / det, (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det, (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det},
        {c02 / det, (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det, (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det}};
    pt_affine r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = static_cast<float>(inv[i][j]);
    float tv[3];
    affine_vector(r, x.t, tv);
    // vec3 unary minus
    for (int i = 0; i < 3; ++i) r.t[i] = -tv[i];
    return r;
}

// Levels of 4-wide nodes under node n (include/gpu_pack.hpp:41-47 counts the same way).
uint32_t tree_depth(const std::vector<pt_bvh_node>& nodes, uint32_t n) {
    if (nodes.empty()) return 0;
    // Iterative: (node, depth) pairs.
    std::vector<std::pair<uint32_t, uint32_t>> work{{n, 1}};
    uint32_t deepest = 0;
    const float inf = std::numeric_limits<float>::infinity();
    while (!work.empty()) {
        auto [k, d] = work.back();
        work.pop_back();
        deepest = std::max(deepest, d);
        for (int c = 0; c < 4; ++c)
            if (nodes[k].count[c] == 0 && nodes[k].lo[0][c] != inf) work.push_back({nodes[k].first[c], d + 1});
    }
    return deepest;
}

}  // namespace pt
