// Repack of a scene description into the device arena (pt_layout.h).
//
// Follows the shape of include/gpu_pack.hpp:57-73 (every tree appended to one
// node array with child indices rebased) but lays leaves out as the
// primitives themselves, in leaf order, so a leaf is one contiguous run of
// 48-byte slots instead of order[] entries pointing into a primitive array.
// Trees not supplied by the caller are built with the library's builder,
// exactly as geometry::build would (include/geometry.hpp:74-104).
#include "scene_host.hpp"

#include <cmath>

#include <algorithm>
#include <cstring>
#include <limits>

namespace pt {

namespace {

float ubits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

bool emits(const pt_material& m) { return m.emission[0] > 0 || m.emission[1] > 0 || m.emission[2] > 0; }

pt_status check_tree(const pt_bvh& t, uint32_t n_prims, const char* what) {
    if (!t.nodes) return PT_OK;
    if (t.n_order != n_prims || (n_prims && !t.order))
        return fail(PT_ERR_INVALID_ARG, std::string(what) + ": order size differs from the primitive count");
    if (n_prims && t.n_nodes == 0) return fail(PT_ERR_INVALID_ARG, std::string(what) + ": no nodes");
    for (uint32_t i = 0; i < t.n_order; ++i)
        if (t.order[i] >= n_prims) return fail(PT_ERR_INVALID_ARG, std::string(what) + ": order entry out of range");
    const float inf = std::numeric_limits<float>::infinity();
    for (uint32_t k = 0; k < t.n_nodes; ++k)
        for (int c = 0; c < 4; ++c) {
            const uint32_t f = t.nodes[k].first[c], n = t.nodes[k].count[c];
            if (n > 0) {
                if (uint64_t(f) + n > t.n_order || n > PT_COUNT_MASK)
                    return fail(PT_ERR_INVALID_ARG, std::string(what) + ": leaf range out of range");
            } else if (t.nodes[k].lo[0][c] != inf && (f >= t.n_nodes || f <= k)) {
                return fail(PT_ERR_INVALID_ARG, std::string(what) + ": child node index out of range");
            }
        }
    return PT_OK;
}

// Appends a tree's nodes, rebased: interior children by node_base, leaves by
// slot_base; leaf count words get PT_LEAF_HAS_SPHERE from has_sphere(slot).
template <class HasSphere>
uint32_t append_nodes(HostArena& A, const std::vector<pt_bvh_node>& nodes, uint32_t slot_base, HasSphere&& has_sphere,
                      uint32_t leaf_flags = 0) {
    if (nodes.empty()) return PT_NONE;
    const uint32_t node_base = uint32_t(A.nodes.size() / 32);
    const float inf = std::numeric_limits<float>::infinity();
    for (const pt_bvh_node& n : nodes) {
        float rec[32];
        // lo[axis][child] then hi[axis][child]: 6 float4, x y z lows then highs
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 4; ++c) {
                rec[4 * a + c] = n.lo[a][c];
                rec[12 + 4 * a + c] = n.hi[a][c];
            }
        for (int c = 0; c < 4; ++c) {
            uint32_t first = n.first[c], count = n.count[c];
            if (count > 0) {
                bool sph = false;
                for (uint32_t k = 0; k < count; ++k) sph |= has_sphere(first + k);
                first += slot_base;
                count |= (sph ? PT_LEAF_HAS_SPHERE : 0u) | leaf_flags;
            } else if (n.lo[0][c] != inf) {
                first += node_base;
            }
            rec[24 + c] = ubits(first);
            rec[28 + c] = ubits(count);
        }
        A.nodes.insert(A.nodes.end(), rec, rec + 32);
    }
    return node_base;
}

void push_tri_slot(HostArena& A, const pt_triangle& t, uint32_t ref) {
    const float s[12] = {t.p0[0], t.p0[1], t.p0[2], t.e1[0], t.e1[1], t.e1[2],
                         t.e2[0], t.e2[1], t.e2[2], ubits(ref), 0, 0};
    A.slots.insert(A.slots.end(), s, s + 12);
}

void push_sphere_slot(HostArena& A, const pt_sphere& sp, uint32_t ref) {
    const float s[12] = {sp.center[0], sp.center[1], sp.center[2], sp.radius, 0, 0, 0, 0,
                         0, ubits(ref | PT_SLOT_SPHERE), 0, 0};
    A.slots.insert(A.slots.end(), s, s + 12);
}

void push_tri_shade(HostArena& A, const pt_triangle& t) {
    PtShadeTri s;
    s.n0_mat = make_float4(t.n0[0], t.n0[1], t.n0[2], ubits(t.material));
    s.n1 = make_float4(t.n1[0], t.n1[1], t.n1[2], 0);
    s.n2 = make_float4(t.n2[0], t.n2[1], t.n2[2], 0);
    s.fn = make_float4(t.face_normal[0], t.face_normal[1], t.face_normal[2], 0);
    A.tri.push_back(s);
    A.tri_uv.insert(A.tri_uv.end(), t.uv, t.uv + 6);
}

// image_texture's constructor (include/texture.hpp:13-21): sRGB bytes to
// linear floats through the same 256-entry table, std::pow in float.
void decode_texture(const pt_texture& t, HostArena& A) {
    float table[256];
    for (int v = 0; v < 256; ++v) {
        const float c = v / 255.0f;
        table[v] = c <= 0.04045f ? c / 12.92f : std::pow((c + 0.055f) / 1.055f, 2.4f);
    }
    const size_t n = 3 * size_t(t.width) * size_t(t.height);
    A.tex.push_back(make_int4(t.width, t.height, int(A.texels.size()), 0));
    for (size_t k = 0; k < n; ++k) A.texels.push_back(table[t.rgb[k]]);
}

}  // namespace

pt_status build_arena(const pt_scene_desc& d, HostArena& A) {
    A = HostArena();
    const uint32_t nm = d.n_materials;
    if (nm && !d.materials) return fail(PT_ERR_INVALID_ARG, "materials: null pointer");
    if ((d.n_spheres && !d.spheres) || (d.n_large_spheres && !d.large_spheres) || (d.n_triangles && !d.triangles) ||
        (d.n_meshes && !d.meshes) || (d.n_instances && !d.instances) || (d.n_lights && !d.lights))
        return fail(PT_ERR_INVALID_ARG, "scene: null array with a nonzero count");
    if (uint64_t(d.n_spheres) + d.n_triangles >= PT_SLOT_SPHERE)
        return fail(PT_ERR_INVALID_ARG, "scene: too many primitives");
    for (uint32_t i = 0; i < nm; ++i)
        if (d.materials[i].type > PT_MAT_DIFFUSE_LIGHT) return fail(PT_ERR_INVALID_ARG, "material: unknown type");
    if (d.n_textures && !d.textures) return fail(PT_ERR_INVALID_ARG, "textures: null pointer");
    uint64_t texels = 0;
    for (uint32_t k = 0; k < d.n_textures; ++k) {
        const pt_texture& t = d.textures[k];
        if (t.width <= 0 || t.height <= 0 || !t.rgb) return fail(PT_ERR_INVALID_ARG, "texture: empty or null image");
        texels += uint64_t(t.width) * uint64_t(t.height);
    }
    if (texels > (1ull << 28)) return fail(PT_ERR_INVALID_ARG, "textures: more than 2^28 texels");
    for (uint32_t i = 0; i < nm; ++i)
        if (d.materials[i].texture > d.n_textures) return fail(PT_ERR_INVALID_ARG, "material: texture out of range");
    auto mat_ok = [&](uint32_t m) { return m < nm; };
    for (uint32_t i = 0; i < d.n_spheres; ++i)
        if (!mat_ok(d.spheres[i].material)) return fail(PT_ERR_INVALID_ARG, "sphere: material out of range");
    for (uint32_t i = 0; i < d.n_large_spheres; ++i)
        if (!mat_ok(d.large_spheres[i].material)) return fail(PT_ERR_INVALID_ARG, "large sphere: material out of range");
    for (uint32_t i = 0; i < d.n_triangles; ++i)
        if (!mat_ok(d.triangles[i].material)) return fail(PT_ERR_INVALID_ARG, "triangle: material out of range");
    for (uint32_t m = 0; m < d.n_meshes; ++m) {
        if (d.meshes[m].n_triangles && !d.meshes[m].triangles) return fail(PT_ERR_INVALID_ARG, "mesh: null triangles");
        for (uint32_t i = 0; i < d.meshes[m].n_triangles; ++i)
            if (!mat_ok(d.meshes[m].triangles[i].material))
                return fail(PT_ERR_INVALID_ARG, "mesh triangle: material out of range");
        if (pt_status st = check_tree(d.meshes[m].tree, d.meshes[m].n_triangles, "mesh tree")) return st;
    }
    for (uint32_t k = 0; k < d.n_instances; ++k) {
        if (d.instances[k].mesh >= d.n_meshes) return fail(PT_ERR_INVALID_ARG, "instance: mesh out of range");
        const uint32_t m = d.instances[k].material;
        if (m != PT_NO_MATERIAL && !mat_ok(m)) return fail(PT_ERR_INVALID_ARG, "instance: material out of range");
    }
    if (d.use_bvh) {
        if (pt_status st = check_tree(d.flat_tree, d.n_spheres + d.n_triangles, "flat tree")) return st;
        if (pt_status st = check_tree(d.instance_tree, d.n_instances, "instance tree")) return st;
    }

    // Materials.
    for (uint32_t i = 0; i < nm; ++i) {
        const pt_material& m = d.materials[i];
        uint32_t flags = emits(m) ? PT_MF_EMITS : 0u;
        if (m.type == PT_MAT_LAMBERTIAN) flags |= PT_MF_DIFFUSE;
        if (m.type == PT_MAT_DIELECTRIC) flags |= PT_MF_TRANSMISSIVE;
        PtMaterial g;
        g.albedo_type = make_float4(m.albedo[0], m.albedo[1], m.albedo[2], ubits(m.type));
        // metal keeps fuzz = f < 1 ? f : 1 (include/material.hpp:83; NaN becomes 1)
        g.emission_fuzz = make_float4(m.emission[0], m.emission[1], m.emission[2], m.fuzz < 1.0f ? m.fuzz : 1.0f);
        // only lambertians are textured (lambertian::texture, include/material.hpp:50)
        const bool textured = m.type == PT_MAT_LAMBERTIAN && m.texture > 0;
        g.ior_flags = make_float4(m.ior, ubits(flags), ubits(textured ? m.texture - 1 : PT_NONE), 0);
        A.has_textures |= textured ? 1 : 0;
        A.mat.push_back(g);
    }
    for (uint32_t k = 0; k < d.n_textures; ++k) decode_texture(d.textures[k], A);

    // Lights: given, or every emissive sphere (include/geometry.hpp:75-77).
    std::vector<uint32_t> lights;
    if (d.lights) {
        lights.assign(d.lights, d.lights + d.n_lights);
        for (uint32_t l : lights)
            if (l >= d.n_spheres) return fail(PT_ERR_INVALID_ARG, "light: sphere out of range");
    } else {
        for (uint32_t i = 0; i < d.n_spheres; ++i)
            if (emits(d.materials[d.spheres[i].material])) lights.push_back(i);
    }
    std::vector<float> power;  // of each light, for the extended pick
    for (uint32_t l : lights) {
        const pt_sphere& s = d.spheres[l];
        const pt_material& m = d.materials[s.material];
        A.lights.push_back({make_float4(s.center[0], s.center[1], s.center[2], s.radius),
                            make_float4(m.emission[0], m.emission[1], m.emission[2], 0)});
        power.push_back(pt_sphere_light_power(pt_light_luminance(m.emission[0], m.emission[1], m.emission[2]),
                                              s.radius));
    }
    // The extended light list adds every emissive triangle of the flat list
    // with a positive area (PT_FLAG_NEE_EXTENDED).
    for (uint32_t i = 0; i < d.n_triangles; ++i) {
        const pt_triangle& t = d.triangles[i];
        const pt_material& m = d.materials[t.material];
        if (!emits(m)) continue;
        const float area = pt_triangle_area(t.e1[0], t.e1[1], t.e1[2], t.e2[0], t.e2[1], t.e2[2]);
        if (!(area > 0.0f) || !(area < 3.0e38f)) continue;
        PtTriLight L;
        L.p0_area = make_float4(t.p0[0], t.p0[1], t.p0[2], area);
        L.e1_er = make_float4(t.e1[0], t.e1[1], t.e1[2], m.emission[0]);
        L.e2_eg = make_float4(t.e2[0], t.e2[1], t.e2[2], m.emission[1]);
        L.fn_eb = make_float4(t.face_normal[0], t.face_normal[1], t.face_normal[2], m.emission[2]);
        A.tri_lights.push_back(L);
        power.push_back(pt_triangle_light_power(pt_light_luminance(m.emission[0], m.emission[1], m.emission[2]), area));
    }
    if (!power.empty()) {
        double total = 0;
        for (float p : power) total += p;
        const size_t n = power.size();
        if (total > 0) {
            A.pick_uniform = float(0.5 / double(n));
            A.pick_power = float(0.5 / total);
        } else {
            A.pick_uniform = float(1.0 / double(n));
            A.pick_power = 0;
        }
        double acc = 0, sum = 0;
        std::vector<double> pick(n);
        for (size_t k = 0; k < n; ++k) sum += pick[k] = double(A.pick_uniform + A.pick_power * power[k]);
        for (size_t k = 0; k < n; ++k) {
            acc += pick[k];
            A.light_cdf.push_back(k + 1 == n ? 1.0f : float(acc / sum));
        }
    }

    for (uint32_t i = 0; i < d.n_large_spheres; ++i) {
        const pt_sphere& s = d.large_spheres[i];
        A.large.push_back(make_float4(s.center[0], s.center[1], s.center[2], s.radius));
        A.large_mat.push_back(s.material);
    }
    for (uint32_t i = 0; i < d.n_spheres; ++i) {
        const pt_sphere& s = d.spheres[i];
        PtShadeSphere g;
        g.cr = make_float4(s.center[0], s.center[1], s.center[2], s.radius);
        g.mat = s.material;
        g.pad0 = g.pad1 = g.pad2 = 0;
        A.sph.push_back(g);
    }
    // Shading triangles: the flat ones, then each mesh's.
    for (uint32_t i = 0; i < d.n_triangles; ++i) push_tri_shade(A, d.triangles[i]);
    std::vector<uint32_t> mesh_tri_base(d.n_meshes);
    for (uint32_t m = 0; m < d.n_meshes; ++m) {
        mesh_tri_base[m] = uint32_t(A.tri.size());
        for (uint32_t i = 0; i < d.meshes[m].n_triangles; ++i) push_tri_shade(A, d.meshes[m].triangles[i]);
    }

    uint32_t depth_flat = 0, depth_inst = 0, depth_mesh = 0;

    // The flat tree over spheres then triangles (include/geometry.hpp:92-97).
    const uint32_t ns = d.n_spheres, nprim = d.n_spheres + d.n_triangles;
    A.flat_root = PT_NONE;
    if (d.use_bvh) {
        std::vector<pt_bvh_node> nodes;
        std::vector<uint32_t> order;
        if (d.flat_tree.nodes) {
            nodes.assign(d.flat_tree.nodes, d.flat_tree.nodes + d.flat_tree.n_nodes);
            order.assign(d.flat_tree.order, d.flat_tree.order + d.flat_tree.n_order);
        } else {
            std::vector<float> boxes(6 * size_t(nprim));
            for (uint32_t i = 0; i < ns; ++i) sphere_box(d.spheres[i].center, d.spheres[i].radius, &boxes[6 * size_t(i)]);
            for (uint32_t i = 0; i < d.n_triangles; ++i) {
                const pt_triangle& t = d.triangles[i];
                triangle_box(t.p0, t.p1, t.p2, &boxes[6 * size_t(ns + i)]);
            }
            build_bvh(boxes.data(), nprim, nodes, order);
        }
        const uint32_t slot_base = uint32_t(A.slots.size() / 12);
        A.flat_root = append_nodes(A, nodes, slot_base, [&](uint32_t k) { return order[k] < ns; });
        for (uint32_t p : order) {
            if (p < ns) push_sphere_slot(A, d.spheres[p], p);
            else push_tri_slot(A, d.triangles[p - ns], p - ns);
        }
        depth_flat = tree_depth(nodes, 0);
        A.n_flat_slots = nprim;
    } else {
        for (uint32_t p = 0; p < ns; ++p) push_sphere_slot(A, d.spheres[p], p);
        for (uint32_t p = 0; p < d.n_triangles; ++p) push_tri_slot(A, d.triangles[p], p);
        A.n_flat_slots = nprim;
    }

    // Each mesh's tree (always built, include/geometry.hpp:78-87) and bounds.
    std::vector<uint32_t> mesh_root(d.n_meshes, PT_NONE);
    std::vector<std::array<float, 6>> mesh_bounds(d.n_meshes);
    for (uint32_t m = 0; m < d.n_meshes; ++m) {
        const pt_mesh& me = d.meshes[m];
        std::vector<float> boxes(6 * size_t(me.n_triangles));
        float b[6] = {std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity(),
                      std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(),
                      -std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity()};
        for (uint32_t i = 0; i < me.n_triangles; ++i) {
            float* bx = &boxes[6 * size_t(i)];
            triangle_box(me.triangles[i].p0, me.triangles[i].p1, me.triangles[i].p2, bx);
            for (int a = 0; a < 3; ++a) {
                b[a] = std::min(b[a], bx[a]);
                b[3 + a] = std::max(b[3 + a], bx[3 + a]);
            }
        }
        std::copy(b, b + 6, mesh_bounds[m].begin());
        std::vector<pt_bvh_node> nodes;
        std::vector<uint32_t> order;
        if (me.tree.nodes) {
            nodes.assign(me.tree.nodes, me.tree.nodes + me.tree.n_nodes);
            order.assign(me.tree.order, me.tree.order + me.tree.n_order);
        } else {
            build_bvh(boxes.data(), me.n_triangles, nodes, order);
        }
        const uint32_t slot_base = uint32_t(A.slots.size() / 12);
        mesh_root[m] = append_nodes(A, nodes, slot_base, [](uint32_t) { return false; });
        for (uint32_t p : order) push_tri_slot(A, me.triangles[p], p);
        depth_mesh = std::max(depth_mesh, tree_depth(nodes, 0));
    }

    // Instances: shading records in instance order; slots in the instance
    // tree's leaf order (or instance order without the BVH).
    for (uint32_t k = 0; k < d.n_instances; ++k) {
        const pt_instance& in = d.instances[k];
        PtShadeInst s;
        for (int r = 0; r < 3; ++r)
            s.row[r] = make_float4(in.to_object.m[r][0], in.to_object.m[r][1], in.to_object.m[r][2], in.to_object.t[r]);
        s.tri_base = mesh_tri_base[in.mesh];
        s.material = in.material;
        s.mesh = in.mesh;
        s.pad = 0;
        A.inst.push_back(s);
    }
    auto push_islot = [&](uint32_t k) {
        const pt_instance& in = d.instances[k];
        float s[16];
        for (int r = 0; r < 3; ++r) {
            s[4 * r + 0] = in.to_object.m[r][0];
            s[4 * r + 1] = in.to_object.m[r][1];
            s[4 * r + 2] = in.to_object.m[r][2];
            s[4 * r + 3] = in.to_object.t[r];
        }
        s[12] = ubits(mesh_root[in.mesh]);
        s[13] = ubits(k);
        s[14] = 0;
        s[15] = 0;
        A.islots.insert(A.islots.end(), s, s + 16);
    };
    A.inst_root = PT_NONE;
    if (d.use_bvh && d.n_instances) {
        std::vector<pt_bvh_node> nodes;
        std::vector<uint32_t> order;
        if (d.instance_tree.nodes) {
            nodes.assign(d.instance_tree.nodes, d.instance_tree.nodes + d.instance_tree.n_nodes);
            order.assign(d.instance_tree.order, d.instance_tree.order + d.instance_tree.n_order);
        } else {
            std::vector<float> boxes(6 * size_t(d.n_instances));
            for (uint32_t k = 0; k < d.n_instances; ++k)
                affine_box(d.instances[k].to_world, mesh_bounds[d.instances[k].mesh].data(), &boxes[6 * size_t(k)]);
            build_bvh(boxes.data(), d.n_instances, nodes, order);
        }
        A.inst_root = append_nodes(A, nodes, 0, [](uint32_t) { return false; }, PT_LEAF_INSTANCES);
        for (uint32_t k : order) push_islot(k);
        depth_inst = tree_depth(nodes, 0);
    } else {
        for (uint32_t k = 0; k < d.n_instances; ++k) push_islot(k);
    }
    for (uint32_t k = 0; k < d.n_instances; ++k)
        if (mesh_root[d.instances[k].mesh] == PT_NONE)
            return fail(PT_ERR_UNSUPPORTED, "instance of an empty mesh");
    A.n_instances = d.n_instances;

    // Stack entries a ray can need: a walk of a tree of D levels holds at
    // most 3D + 1; a mesh walk runs on top of the instance walk.
    uint32_t need = depth_flat ? 3 * depth_flat + 1 : 0;
    if (d.n_instances) need = std::max(need, 3 * (depth_inst + depth_mesh) + 1);
    A.stack_entries = need;
    A.max_depth = std::max(depth_flat, std::max(depth_inst, depth_mesh));
    if (need > PT_STACK_MAX)
        return fail(PT_ERR_STACK_OVERFLOW, "scene: a traversal could need " + std::to_string(need) +
                                               " stack entries, more than the " + std::to_string(PT_STACK_MAX) +
                                               " the kernels hold");
    A.sky = d.sky;
    A.sample_lights = d.sample_lights;
    A.use_bvh = d.use_bvh;
    A.n_spheres = d.n_spheres;
    return PT_OK;
}

int ordered_boxes(const std::vector<float>& nodes) {
    for (size_t k = 0; k + 32 <= nodes.size(); k += 32)
        for (int i = 0; i < 12; ++i)
            if (!(nodes[k + i] <= nodes[k + 12 + i])) return 0;
    return 1;
}

uint32_t tree_kib(const std::vector<float>& nodes, const std::vector<float>& slots) {
    const uint64_t kib = (uint64_t(nodes.size()) + uint64_t(slots.size())) * sizeof(float) / 1024;
    return kib > 0xffffffffu ? 0xffffffffu : uint32_t(kib);
}

// Checked over every tree of the arena (conservative: the packed entries are
// only used by walks of a flat tree, which push flat-tree entries alone).
int stack_pack8(const std::vector<float>& nodes) {
    if (nodes.size() / 32 >= (size_t(1) << 31)) return 0;
    for (size_t k = 0; k + 32 <= nodes.size(); k += 32)
        for (int c = 0; c < 4; ++c) {
            uint32_t first, count;
            std::memcpy(&first, &nodes[k + 24 + c], 4);
            std::memcpy(&count, &nodes[k + 28 + c], 4);
            if (count == 0) {
                if (first >= 0x80000000u) return 0;
            } else if ((count & PT_COUNT_MASK) > 15u || first >= (1u << 26)) {
                return 0;
            }
        }
    return 1;
}

}  // namespace pt
