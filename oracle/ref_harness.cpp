// ref_harness.cpp -- TEST INFRASTRUCTURE, not part of the product.
//
// Drives the reference implementation itself: compiled by oracle/build_ref.py
// against photon_tracer's own headers where they lie (include/*.hpp of the
// reference checkout), with the reference's Makefile flags (-O3 -std=c++17,
// no -march) plus -ffp-contract=off, into oracle/_ref/libptref.so. Used by the
// tests to pin the CPU restatement (pt_oracle.c) and the library's BVH
// builder, and by bench.py as the reference CPU baseline.
//
// Only public members of the reference are used. Where the reference keeps a
// value private (geometry::hit's choice of primitive, the camera's aspect),
// the harness re-composes it from public pieces and cross-checks the result
// against the reference's own call.
#include <array>
#include <atomic>
#include <cstring>
#include <map>
#include <fstream>
#include <sstream>
#include <thread>
#include <vector>

#include "image_write.hpp"
#include "renderer.hpp"
#include "../include/photon_cuda.h"
#include "../include/photon_cuda_geometry.hpp"

namespace {

struct ref_scene {
    geometry world;
    std::vector<const material*> mats;
};

// The reference's own image_texture over a pt_texture's sRGB bytes.
std::shared_ptr<const image_texture> texture_from(const pt_texture& t) {
    image8 img;
    img.width = t.width;
    img.height = t.height;
    img.rgb.assign(t.rgb, t.rgb + 3 * size_t(t.width) * size_t(t.height));
    return std::make_shared<const image_texture>(img);
}

std::shared_ptr<material> material_from(const pt_material& m,
                                        const std::vector<std::shared_ptr<const image_texture>>& textures) {
    const color albedo(m.albedo[0], m.albedo[1], m.albedo[2]);
    switch (m.type) {
        case PT_MAT_LAMBERTIAN:
            return std::make_shared<lambertian>(albedo, m.texture > 0 ? textures[m.texture - 1] : nullptr);
        case PT_MAT_METAL: return std::make_shared<metal>(albedo, m.fuzz);
        case PT_MAT_DIELECTRIC: return std::make_shared<dielectric>(m.ior);
        default: return std::make_shared<diffuse_light>(color(m.emission[0], m.emission[1], m.emission[2]));
    }
}

point3 P(const float* p) { return point3(p[0], p[1], p[2]); }

triangle make_tri(const pt_triangle& t, const material* m) {
    // The reference's smooth constructor from the corners as given.
    triangle tr(P(t.p0), P(t.p1), P(t.p2), P(t.n0), P(t.n1), P(t.n2), m);
    for (int k = 0; k < 6; ++k) tr.uv[k] = t.uv[k];
    return tr;
}

// The camera with its four fields set (the reference's constructor fixes the
// aspect at 16:9). camera is a standard-layout class of four vec3 in the
// order origin, lower_left_corner, horizontal, vertical; the accessors check
// the copy landed where they read.
camera camera_from(const pt_camera* c) {
    static_assert(sizeof(camera) == 12 * sizeof(float), "camera layout");
    camera cam;
    float f[12];
    std::memcpy(f, c->origin, 12);
    std::memcpy(f + 3, c->lower_left, 12);
    std::memcpy(f + 6, c->horizontal, 12);
    std::memcpy(f + 9, c->vertical, 12);
    std::memcpy(static_cast<void*>(&cam), f, sizeof(f));
    return cam;
}

}  // namespace

extern "C" {

// Builds the reference geometry for desc (trees built by geometry::build).
void* ref_scene_create(const pt_scene_desc* d) {
    auto* s = new ref_scene();
    geometry& w = s->world;
    std::vector<std::shared_ptr<const image_texture>> textures;
    for (uint32_t k = 0; k < d->n_textures; ++k) textures.push_back(texture_from(d->textures[k]));
    for (uint32_t i = 0; i < d->n_materials; ++i) s->mats.push_back(w.own(material_from(d->materials[i], textures)));
    for (uint32_t i = 0; i < d->n_spheres; ++i) {
        const pt_sphere& sp = d->spheres[i];
        w.spheres.emplace_back(P(sp.center), sp.radius, s->mats[sp.material]);
    }
    for (uint32_t i = 0; i < d->n_large_spheres; ++i) {
        const pt_sphere& sp = d->large_spheres[i];
        w.large_spheres.emplace_back(P(sp.center), sp.radius, s->mats[sp.material]);
    }
    for (uint32_t i = 0; i < d->n_triangles; ++i)
        w.triangles.push_back(make_tri(d->triangles[i], s->mats[d->triangles[i].material]));
    for (uint32_t m = 0; m < d->n_meshes; ++m) {
        std::vector<triangle> tris;
        for (uint32_t i = 0; i < d->meshes[m].n_triangles; ++i)
            tris.push_back(make_tri(d->meshes[m].triangles[i], s->mats[d->meshes[m].triangles[i].material]));
        w.add_mesh(std::move(tris));
    }
    for (uint32_t k = 0; k < d->n_instances; ++k) {
        const pt_instance& in = d->instances[k];
        affine x;
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c) x.m[r][c] = in.to_world.m[r][c];
            x.t.e[r] = in.to_world.t[r];
        }
        w.add_instance(in.mesh, x, in.material == PT_NO_MATERIAL ? nullptr : s->mats[in.material]);
    }
    w.sky = d->sky != 0;
    w.sample_lights = d->sample_lights != 0;
    w.build(d->use_bvh != 0);
    return s;
}

void ref_scene_destroy(void* h) { delete static_cast<ref_scene*>(h); }

// Copies the fields the reference's constructors computed, for comparison
// with the description (e1, e2, face normal per triangle; to_object per instance).
void ref_triangle_fields(void* h, int mesh, uint32_t i, float out[12]) {
    const geometry& w = static_cast<ref_scene*>(h)->world;
    const triangle& t = mesh < 0 ? w.triangles[i] : w.meshes[mesh].triangles[i];
    const vec3 v[4] = {t.p0, t.e1, t.e2, t.face_normal};
    for (int k = 0; k < 4; ++k)
        for (int a = 0; a < 3; ++a) out[3 * k + a] = v[k].e[a];
}

void ref_instance_to_object(void* h, uint32_t k, float out[12]) {
    const geometry& w = static_cast<ref_scene*>(h)->world;
    const affine& x = w.instances[k].to_object;
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) out[3 * r + c] = x.m[r][c];
        out[9 + r] = x.t.e[r];
    }
}

// A tree the reference built: which 0 = flat, 1 = instances, 2 = mesh `mesh`.
// Returns the node count; copies when the buffers are large enough.
uint32_t ref_tree(void* h, int which, int mesh, pt_bvh_node* nodes, uint32_t cap_nodes, uint32_t* order,
                  uint32_t cap_order, uint32_t* n_order) {
    const geometry& w = static_cast<ref_scene*>(h)->world;
    const bvh& t = which == 0 ? w.flat_tree() : which == 1 ? w.instances_tree() : w.meshes[mesh].tree;
    static_assert(sizeof(bvh::node) == sizeof(pt_bvh_node), "node layout");
    if (nodes && cap_nodes >= t.nodes.size()) std::memcpy(nodes, t.nodes.data(), t.nodes.size() * sizeof(pt_bvh_node));
    if (order && cap_order >= t.order.size()) std::memcpy(order, t.order.data(), t.order.size() * sizeof(uint32_t));
    *n_order = uint32_t(t.order.size());
    return uint32_t(t.nodes.size());
}

// geometry::hit's choice of primitive, re-composed from the public trees with
// the lambdas of geometry.hpp:117-139 and hit_instance :212-229, and checked
// against geometry::hit itself: *mismatch counts rays where rec.t or rec.p differ.
void ref_trace_closest(void* h, const float* rays, size_t n, float t_min, float t_max_in, pt_hit* out,
                       uint64_t* mismatch) {
    const geometry& w = static_cast<ref_scene*>(h)->world;
    uint64_t bad = 0;
    for (size_t q = 0; q < n; ++q) {
        const float* rr = rays + 6 * q;
        const ray r(point3(rr[0], rr[1], rr[2]), vec3(rr[3], rr[4], rr[5]));
        real t_max = t_max_in;
        uint32_t kind = PT_HIT_NONE, index = 0, sub = 0;
        real u = 0, v = 0;
        for (uint32_t i = 0; i < w.large_spheres.size(); ++i)
            if (w.large_spheres[i].intersect<double>(r, t_min, t_max)) { kind = PT_HIT_LARGE; index = i; }
        const uint32_t ns = uint32_t(w.spheres.size());
        auto test = [&](uint32_t p, real& t_far) {
            if (p < ns) {
                if (w.spheres[p].intersect(r, t_min, t_far)) { kind = PT_HIT_SPHERE; index = p; }
            } else if (w.triangles[p - ns].intersect(r, t_min, t_far, u, v)) {
                kind = PT_HIT_TRIANGLE; index = p - ns;
            }
        };
        auto test_instance = [&](uint32_t k, real& t_far) {
            const geometry::instance& in = w.instances[k];
            const geometry::mesh& m = w.meshes[in.mesh];
            const ray local(in.to_object.point(r.origin()), in.to_object.vector(r.direction()));
            bool found = false;
            real ht = t_far, hu = 0, hv = 0;
            uint32_t tri = 0;
            m.tree.traverse(local, t_min, ht, [&](uint32_t ti, real& t_mesh) {
                if (m.triangles[ti].intersect(local, t_min, t_mesh, hu, hv)) { found = true; tri = ti; }
            });
            if (found) { kind = PT_HIT_INSTANCE; index = k; t_far = ht; u = hu; v = hv; sub = tri; }
        };
        if (w.uses_bvh()) {
            w.flat_tree().traverse(r, t_min, t_max, test);
            if (!w.instances.empty()) w.instances_tree().traverse(r, t_min, t_max, test_instance);
        } else {
            const uint32_t np = ns + uint32_t(w.triangles.size());
            for (uint32_t p = 0; p < np; ++p) test(p, t_max);
            for (uint32_t k = 0; k < w.instances.size(); ++k) test_instance(k, t_max);
        }
        hit_record rec;
        const bool got = w.hit(r, t_min, t_max_in, rec);
        if (got != (kind != PT_HIT_NONE)) ++bad;
        else if (got) {
            const point3 p = r.at(t_max);
            if (rec.t != t_max || rec.p.e[0] != p.e[0] || rec.p.e[1] != p.e[1] || rec.p.e[2] != p.e[2]) ++bad;
        }
        out[q].kind = kind;
        out[q].index = kind == PT_HIT_NONE ? 0 : index;
        out[q].sub = sub;
        out[q].t = t_max;
        out[q].u = u;
        out[q].v = v;
    }
    *mismatch = bad;
}

void ref_trace_any(void* h, const float* rays, size_t n, float t_min, float t_max, uint8_t* out) {
    const geometry& w = static_cast<ref_scene*>(h)->world;
    for (size_t q = 0; q < n; ++q) {
        const float* rr = rays + 6 * q;
        out[q] = w.occluded(ray(point3(rr[0], rr[1], rr[2]), vec3(rr[3], rr[4], rr[5])), t_min, t_max) ? 1 : 0;
    }
}

// render_row_linear over scanlines [row0, row0 + rows) on `threads` threads
// taking rows from an atomic counter (src/main.cpp:137-158), written in
// pt_render's layout (top row first; aux 7 floats or NULL). Returns the ray
// count (include/renderer.hpp:19, summed as main.cpp:157 does).
uint64_t ref_render(void* h, const pt_camera* c, int W, int H, int spp, int depth, uint64_t seed, int first_sample,
                    int row0, int rows, float* out, float* aux, int threads) {
    const geometry& w = static_cast<ref_scene*>(h)->world;
    const camera cam = camera_from(c);
    std::atomic<int> next{row0};
    std::atomic<long long> total{0};
    auto worker = [&]() {
        rays_traced = 0;
        for (int j = next.fetch_add(1); j < row0 + rows; j = next.fetch_add(1)) {
            const size_t row = size_t(H - 1 - j) * W;
            render_row_linear(w, cam, j, W, H, spp, depth, out + 3 * row, seed, first_sample,
                              aux ? aux + aux_floats * row : nullptr);
        }
        total += rays_traced;
    };
    if (threads <= 1) {
        worker();
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
    }
    return uint64_t(total.load());
}

// render_row_impl's loop (include/renderer.hpp:370-396) with the reference's
// own seed_row stream, capturing thread_rng's state before each ray_color:
// states gets 4 words per (pixel, sample), pixels row by row from j = row0,
// as PT_RNG_SNAPSHOT reads them. Writes the image like ref_render.
uint64_t ref_render_snapshot(void* h, const pt_camera* c, int W, int H, int spp, int depth, uint64_t seed,
                             int first_sample, int row0, int rows, float* out, float* aux, uint64_t* states) {
    const geometry& w = static_cast<ref_scene*>(h)->world;
    const camera cam = camera_from(c);
    rays_traced = 0;
    for (int j = row0; j < row0 + rows; ++j) {
        seed_row(seed, j, first_sample);
        const real scale = real(1) / spp;
        for (int i = 0; i < W; ++i) {
            color pc(0, 0, 0), albedo(0, 0, 0);
            vec3 normal(0, 0, 0);
            real lum2 = 0;
            for (int s = 0; s < spp; ++s) {
                begin_sample(seed, i, j, static_cast<uint32_t>(first_sample + s));
                real du, dv;
                sample_2d(0, du, dv);
                const ray r = cam.get_ray((i + du) / (W - 1), (j + dv) / (H - 1));
                std::memcpy(states + 4 * ((size_t(j - row0) * W + i) * spp + s), thread_rng.s, 32);
                first_hit first;
                const color col = ray_color<true>(r, w, depth, &first);
                pc = pc + col;
                albedo = albedo + first.albedo;
                normal = normal + first.normal;
                lum2 += luminance(col) * luminance(col);
            }
            const size_t px = size_t(H - 1 - j) * W + i;
            for (int k = 0; k < 3; ++k) out[3 * px + k] = static_cast<float>(pc.e[k] * scale);
            if (aux) {
                for (int k = 0; k < 3; ++k) {
                    aux[7 * px + k] = static_cast<float>(albedo.e[k] * scale);
                    aux[7 * px + 3 + k] = static_cast<float>(normal.e[k] * scale);
                }
                aux[7 * px + 6] = static_cast<float>(lum2 * scale);
            }
        }
    }
    return uint64_t(rays_traced);
}

// The reference's denoiser (include/denoise.hpp:55-139).
void ref_denoise(int w, int h, const float* color, const float* albedo, const float* normal, const float* variance,
                 float* out, int threads) {
    denoise({w, h, color, albedo, normal, variance}, out, threads);
}

// The reference's sampler, for known-answer checks: (a, b) of pair_offset
// at the given bounce (-1: before any set_bounce) for sample index of pixel (i, j).
void ref_sample_2d(uint64_t seed, int i, int j, uint32_t index, int bounce, int pair_offset, float out[2]) {
    begin_sample(seed, i, j, index);
    if (bounce >= 0) set_bounce(bounce);
    thread_rng.seed(1);
    real a, b;
    sample_2d(pair_offset, a, b);
    out[0] = a;
    out[1] = b;
}

// The camera the reference builds (16:9) for a lookfrom/lookat/vfov.
void ref_camera(const float from[3], const float at[3], double vfov, pt_camera* out) {
    const camera c(point3(from[0], from[1], from[2]), point3(at[0], at[1], at[2]), vfov);
    for (int a = 0; a < 3; ++a) {
        out->origin[a] = c.position().e[a];
        out->lower_left[a] = c.corner().e[a];
        out->horizontal[a] = c.across().e[a];
        out->vertical[a] = c.up().e[a];
    }
}

// Checks make_camera's layout assumption: the accessors of the copied camera.
int ref_camera_roundtrip(const pt_camera* c) {
    const camera cam = camera_from(c);
    for (int a = 0; a < 3; ++a)
        if (cam.position().e[a] != c->origin[a] || cam.corner().e[a] != c->lower_left[a] ||
            cam.across().e[a] != c->horizontal[a] || cam.up().e[a] != c->vertical[a])
            return 0;
    return 1;
}

// The reference's own scenes, for comparing with the library's generators:
// fills counts {spheres, large, triangles, materials} and copies spheres
// (center, radius) and triangles (p0, e1, e2) when buffers are given.
void ref_builtin_scene(int id, uint32_t counts[4], float* spheres, float* tris) {
    const geometry w = build_world(static_cast<scene_id>(id), true);
    counts[0] = uint32_t(w.spheres.size());
    counts[1] = uint32_t(w.large_spheres.size());
    counts[2] = uint32_t(w.triangles.size());
    counts[3] = 0;
    if (spheres)
        for (size_t i = 0; i < w.spheres.size(); ++i) {
            for (int a = 0; a < 3; ++a) spheres[4 * i + a] = w.spheres[i].center.e[a];
            spheres[4 * i + 3] = w.spheres[i].radius;
        }
    if (tris)
        for (size_t i = 0; i < w.triangles.size(); ++i)
            for (int a = 0; a < 3; ++a) {
                tris[9 * i + a] = w.triangles[i].p0.e[a];
                tris[9 * i + 3 + a] = w.triangles[i].e1.e[a];
                tris[9 * i + 6 + a] = w.triangles[i].e2.e[a];
            }
}

}  // extern "C"

extern "C" {
// The reference's write_image (include/image_write.hpp:15-33).
int ref_write_image(const char* path, int w, int h, const float* linear) { return write_image(path, w, h, linear) ? 1 : 0; }
}

extern "C" {
// The reference's own worlds as its CLI builds them (src/main.cpp:63-108):
// build_world(id, use_bvh, the OBJ's text, a reader for the files beside it,
// turn, crowd side, flatten) with NEE on, exported in the C ABI's layout by
// photon_cuda_geometry.hpp (the trees geometry::build made included), with
// make_camera(id). For writing fixtures of the reference's OBJ scenes (the
// teapot, the crowd and its flattened form, the spot crowd).
struct ref_world {
    geometry world;
    photon_cuda::scene_arrays arrays;
    pt_camera cam;
};

static std::string read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return std::string();
    std::ostringstream buf;
    buf << f.rdbuf();
    return buf.str();
}

void* ref_world_create(int id, const char* obj_path, int crowd_side, int flatten, double turn_deg) {
    const std::string path = obj_path ? obj_path : "";
    const std::string dir = path.find('/') == std::string::npos ? "" : path.substr(0, path.find_last_of('/') + 1);
    const std::string text = path.empty() ? std::string() : read_file(path);
    const file_reader beside = [dir](const std::string& name) { return read_file(dir + name); };
    auto* w = new ref_world();
    const scene_id sid = static_cast<scene_id>(id);
    w->world = build_world(sid, sid != scene_id::materials, text, beside, turn_deg, crowd_side, flatten != 0);
    w->world.sample_lights = true;
    w->arrays.from(w->world);
    w->cam = photon_cuda::camera_of(make_camera(sid));
    return w;
}

const pt_scene_desc* ref_world_desc(void* h) { return &static_cast<ref_world*>(h)->arrays.desc; }
const pt_camera* ref_world_camera(void* h) { return &static_cast<ref_world*>(h)->cam; }
void ref_world_destroy(void* h) { delete static_cast<ref_world*>(h); }
}  // extern "C"

// ---- the room-mesh benchmark frame, built through the reference's own API ----------------
// A restatement, in the reference's classes and float arithmetic, of this
// project's room-mesh generator (the closed room without a front wall, a
// ceiling lamp, a glass sphere and a radially displaced icosphere with
// area-weighted vertex normals, include/obj.hpp:198-204), so the reference
// arm of the benchmark renders the frame without loading any product code.
// tests/test_ref_arm.py checks it equal, byte for byte, to the product's
// generated description.
namespace {
uint32_t rm_hash32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
double rm_lattice(int i, int j, int k, uint32_t seed) {
    uint32_t h = rm_hash32(seed ^ 0x9e3779b9u);
    h = rm_hash32(h ^ uint32_t(i) * 0x8da6b343u);
    h = rm_hash32(h ^ uint32_t(j) * 0xd8163841u);
    h = rm_hash32(h ^ uint32_t(k) * 0xcb1ab31fu);
    return (h >> 8) * (2.0 / 16777216.0) - 1.0;
}
double rm_noise(double x, double y, double z, uint32_t seed) {
    const double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    const int ix = int(fx), iy = int(fy), iz = int(fz);
    auto s = [](double t) { return t * t * (3 - 2 * t); };
    const double tx = s(x - fx), ty = s(y - fy), tz = s(z - fz);
    double acc = 0;
    for (int c = 0; c < 8; ++c) {
        const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
        acc += (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz) * rm_lattice(ix + dx, iy + dy, iz + dz, seed);
    }
    return acc;
}
double rm_fbm4(double x, double y, double z, uint32_t seed) {
    double sum = 0, amp = 1, f = 2.0;
    for (int o = 0; o < 4; ++o) {
        sum += amp * rm_noise(x * f, y * f, z * f, seed + 101u * uint32_t(o));
        amp *= 0.5;
        f *= 2;
    }
    return sum;
}
point3 rm_p(double x, double y, double z) { return point3(float(x), float(y), float(z)); }

void room_mesh_world(geometry& w, uint64_t seed, int subdiv) {
    w.sky = false;
    const material* white = w.own(std::make_shared<lambertian>(color(0.73f, 0.73f, 0.73f)));
    const material* red = w.own(std::make_shared<lambertian>(color(0.65f, 0.05f, 0.05f)));
    const material* green = w.own(std::make_shared<lambertian>(color(0.12f, 0.45f, 0.15f)));
    add_quad(w, rm_p(-1, -1, 1), rm_p(2, 0, 0), rm_p(0, 0, -2), white);
    add_quad(w, rm_p(-1, 1, 1), rm_p(2, 0, 0), rm_p(0, 0, -2), white);
    add_quad(w, rm_p(-1, -1, -1), rm_p(2, 0, 0), rm_p(0, 2, 0), white);
    add_quad(w, rm_p(-1, -1, 1), rm_p(0, 0, -2), rm_p(0, 2, 0), red);
    add_quad(w, rm_p(1, -1, 1), rm_p(0, 0, -2), rm_p(0, 2, 0), green);
    w.spheres.emplace_back(rm_p(0, 0.82, -0.1), 0.15f, w.own(std::make_shared<diffuse_light>(color(15, 15, 15))));
    w.spheres.emplace_back(rm_p(0.5, -0.8, 0.35), 0.2f, w.own(std::make_shared<dielectric>(1.5f)));
    // icosphere: 12 corners, then midpoints pushed out to the unit sphere, in double
    std::vector<std::array<double, 3>> v;
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    const double base[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                                {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& p : base) {
        const double l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        v.push_back({p[0] / l, p[1] / l, p[2] / l});
    }
    std::vector<std::array<uint32_t, 3>> f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11},
                                              {1, 5, 9}, {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                              {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8}, {3, 8, 9},
                                              {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (int s = 0; s < subdiv; ++s) {
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> mid;
        auto midpoint = [&](uint32_t a, uint32_t b) {
            const auto key = std::make_pair(std::min(a, b), std::max(a, b));
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            double p[3];
            for (int k = 0; k < 3; ++k) p[k] = 0.5 * (v[a][k] + v[b][k]);
            const double l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
            v.push_back({p[0] / l, p[1] / l, p[2] / l});
            mid.emplace(key, uint32_t(v.size() - 1));
            return uint32_t(v.size() - 1);
        };
        std::vector<std::array<uint32_t, 3>> next;
        for (const auto& q : f) {
            const uint32_t a = midpoint(q[0], q[1]), b = midpoint(q[1], q[2]), c = midpoint(q[2], q[0]);
            next.push_back({q[0], a, c});
            next.push_back({q[1], b, a});
            next.push_back({q[2], c, b});
            next.push_back({a, b, c});
        }
        f.swap(next);
    }
    // radial displacement: radius 0.45 * (1 + (0.05 / 0.45) * fbm4(direction)) about (-0.2, -0.5, -0.25)
    const double center[3] = {-0.2, -0.5, -0.25}, radius = 0.45, amp = 0.05 / 0.45;
    std::vector<point3> pos;
    for (auto& p : v) {
        const double r = radius * (1.0 + amp * rm_fbm4(p[0], p[1], p[2], static_cast<uint32_t>(seed)));
        pos.push_back(rm_p(center[0] + r * p[0], center[1] + r * p[1], center[2] + r * p[2]));
    }
    std::vector<vec3> acc(pos.size(), vec3(0, 0, 0));
    for (const auto& q : f) {
        const vec3 n = cross(pos[q[1]] - pos[q[0]], pos[q[2]] - pos[q[0]]);
        for (int k = 0; k < 3; ++k) acc[q[k]] = acc[q[k]] + n;
    }
    const material* clay = w.own(std::make_shared<lambertian>(color(0.8f, 0.8f, 0.8f)));
    for (const auto& q : f)
        w.triangles.emplace_back(pos[q[0]], pos[q[1]], pos[q[2]], acc[q[0]].normalize(), acc[q[1]].normalize(),
                                 acc[q[2]].normalize(), clay);
}

// camera.hpp:18-34 with the aspect ratio a parameter (1 for the square frame).
camera square_camera(point3 from, point3 at, double vfov_deg, double aspect) {
    const double viewport_height = 2.0 * std::tan(vfov_deg * M_PI / 360.0);
    const double viewport_width = aspect * viewport_height;
    const vec3 w = (from - at).normalize();
    const vec3 u = cross(vec3(0, 1, 0), w).normalize();
    const vec3 v = cross(w, u);
    pt_camera c;
    const vec3 horizontal = u * viewport_width, vertical = v * viewport_height;
    const point3 llc = from - (horizontal * 0.5) - (vertical * 0.5) - w;
    for (int a = 0; a < 3; ++a) {
        c.origin[a] = from.e[a];
        c.lower_left[a] = llc.e[a];
        c.horizontal[a] = horizontal.e[a];
        c.vertical[a] = vertical.e[a];
    }
    return camera_from(&c);
}
}  // namespace

extern "C" {
// The room-mesh frame's scene (icosphere subdivision `subdiv`, noise seed
// `seed`) and its camera (from (0, 0, 3.3) at the origin, vfov 40, square),
// built by the reference's geometry::build with its BVH.
void* ref_room_mesh_world(uint64_t seed, int subdiv) {
    auto* w = new ref_world();
    room_mesh_world(w->world, seed, subdiv);
    w->world.sample_lights = true;
    w->world.build(true);
    w->arrays.from(w->world);
    w->cam = photon_cuda::camera_of(square_camera(rm_p(0, 0, 3.3), rm_p(0, 0, 0), 40.0, 1.0));
    return w;
}

// render_row_linear over the listed scanlines (j counted from the bottom)
// on `threads` threads taking rows from an atomic counter (src/main.cpp:137-158);
// out gets each row at its place in a W x H frame (top row first) or is
// NULL. Returns the ray count.
uint64_t ref_world_render_rows(void* h, int W, int H, int spp, int depth, uint64_t seed, const int* rows,
                               int n_rows, float* out, int threads) {
    const ref_world* rw = static_cast<ref_world*>(h);
    const camera cam = camera_from(&rw->cam);
    std::atomic<int> next{0};
    std::atomic<long long> total{0};
    auto worker = [&]() {
        rays_traced = 0;
        std::vector<float> row(3 * size_t(W));
        for (int k = next.fetch_add(1); k < n_rows; k = next.fetch_add(1)) {
            const int j = rows[k];
            float* dst = out ? out + 3 * size_t(H - 1 - j) * W : row.data();
            render_row_linear(rw->world, cam, j, W, H, spp, depth, dst, seed, 0, nullptr);
        }
        total += rays_traced;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    return uint64_t(total.load());
}
}  // extern "C"
