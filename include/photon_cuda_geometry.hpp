// photon_cuda_geometry.hpp -- header-only bridge from photon_tracer's scene
// API to libphoton_cuda.
//
// Include it after photon_tracer's renderer.hpp (it uses class geometry,
// camera and the material classes). It converts a built geometry into a
// pt_scene_desc -- primitives, materials (mapped by dynamic_cast, as
// include/gpu_pack.hpp:89-113 maps them), instances, the light list and the
// trees geometry::build made (bvh::node is byte-compatible with pt_bvh_node)
// -- and wraps the frame render in the signature of the CPU row loop
// (src/main.cpp:146-158 around render_row_linear, include/renderer.hpp:411-416).
//
//   geometry world = build_world(scene_id::room, true);
//   photon_cuda::gpu_scene gpu;
//   if (gpu.upload(world) != PT_OK) fail(pt_last_error());
//   gpu.render(cam, W, H, spp, 10, image.data(), seed, 0, aux_or_null, &rays);
//
// Textured lambertians carry their texture's sRGB image (texture.hpp) and
// the triangles their texture coordinates; the desc points into the
// geometry's own images, so the geometry must outlive the upload.
#pragma once

#include <cstring>
#include <map>
#include <vector>

#include "photon_cuda.h"

namespace photon_cuda {

static_assert(sizeof(pt_bvh_node) == 128, "pt_bvh_node is bvh::node");

// The four camera fields (include/camera.hpp:39-42).
inline pt_camera camera_of(const camera& cam) {
    pt_camera c;
    for (int a = 0; a < 3; ++a) {
        c.origin[a] = cam.position().e[a];
        c.lower_left[a] = cam.corner().e[a];
        c.horizontal[a] = cam.across().e[a];
        c.vertical[a] = cam.up().e[a];
    }
    return c;
}

// The arrays of one geometry in the C ABI's layout; owns them.
struct scene_arrays {
    std::vector<pt_material> materials;
    std::vector<pt_sphere> spheres, large;
    std::vector<pt_triangle> triangles;
    std::vector<std::vector<pt_triangle>> mesh_tris;
    std::vector<pt_mesh> meshes;
    std::vector<pt_instance> instances;
    std::vector<uint32_t> lights;
    std::vector<pt_texture> textures;  // point into the geometry's textures (kept alive by it)
    pt_scene_desc desc;

    // Fills the arrays and desc from a built geometry.
    void from(const geometry& world) {
        std::map<const material*, uint32_t> index;
        std::map<const image_texture*, uint32_t> tex_index;
        // a texture's sRGB image, once per texture (lambertian::texture, texture.hpp:36-38);
        // materials refer to textures[k] as k + 1
        auto tex = [&](const image_texture* t) -> uint32_t {
            auto found = tex_index.find(t);
            if (found != tex_index.end()) return found->second;
            pt_texture pt;
            pt.width = t->source.width;
            pt.height = t->source.height;
            pt.rgb = t->source.rgb.data();
            const uint32_t k = uint32_t(textures.size()) + 1;
            textures.push_back(pt);
            tex_index.emplace(t, k);
            return k;
        };
        auto mat = [&](const material* m) -> uint32_t {
            if (!m) return PT_NO_MATERIAL;
            auto found = index.find(m);
            if (found != index.end()) return found->second;
            pt_material p;
            std::memset(&p, 0, sizeof(p));
            p.ior = 1.5f;
            p.texture = 0;
            if (auto* l = dynamic_cast<const lambertian*>(m)) {
                p.type = PT_MAT_LAMBERTIAN;
                for (int a = 0; a < 3; ++a) p.albedo[a] = l->albedo.e[a];
                if (l->texture) p.texture = tex(l->texture.get());
            } else if (auto* me = dynamic_cast<const metal*>(m)) {
                p.type = PT_MAT_METAL;
                for (int a = 0; a < 3; ++a) p.albedo[a] = me->albedo.e[a];
                p.fuzz = me->fuzz;
            } else if (auto* d = dynamic_cast<const dielectric*>(m)) {
                p.type = PT_MAT_DIELECTRIC;
                p.ior = d->ior;
            } else {
                p.type = PT_MAT_DIFFUSE_LIGHT;
            }
            for (int a = 0; a < 3; ++a) p.emission[a] = m->emission.e[a];
            const uint32_t k = uint32_t(materials.size());
            materials.push_back(p);
            index.emplace(m, k);
            return k;
        };
        auto sph = [&](const sphere& s) {
            pt_sphere p;
            for (int a = 0; a < 3; ++a) p.center[a] = s.center.e[a];
            p.radius = s.radius;
            p.material = mat(s.mat);
            return p;
        };
        auto tri = [&](const triangle& t) {
            pt_triangle p;
            const vec3* src[9] = {&t.p0, &t.e1, &t.e2, &t.n0, &t.n1, &t.n2, &t.face_normal, &t.p1, &t.p2};
            float* dst[9] = {p.p0, p.e1, p.e2, p.n0, p.n1, p.n2, p.face_normal, p.p1, p.p2};
            for (int k = 0; k < 9; ++k)
                for (int a = 0; a < 3; ++a) dst[k][a] = src[k]->e[a];
            p.material = mat(t.mat);
            for (int k = 0; k < 6; ++k) p.uv[k] = t.uv[k];
            return p;
        };
        auto tree = [](const bvh& b) {
            pt_bvh t;
            t.nodes = reinterpret_cast<const pt_bvh_node*>(b.nodes.data());
            t.n_nodes = uint32_t(b.nodes.size());
            t.order = b.order.data();
            t.n_order = uint32_t(b.order.size());
            return t;
        };
        for (const sphere& s : world.spheres) spheres.push_back(sph(s));
        for (const sphere& s : world.large_spheres) large.push_back(sph(s));
        for (const triangle& t : world.triangles) triangles.push_back(tri(t));
        for (const auto& m : world.meshes) {
            mesh_tris.emplace_back();
            for (const triangle& t : m.triangles) mesh_tris.back().push_back(tri(t));
        }
        for (size_t m = 0; m < world.meshes.size(); ++m) {
            pt_mesh pm;
            pm.triangles = mesh_tris[m].data();
            pm.n_triangles = uint32_t(mesh_tris[m].size());
            pm.tree = tree(world.meshes[m].tree);
            meshes.push_back(pm);
        }
        for (const auto& in : world.instances) {
            pt_instance p;
            p.mesh = in.mesh;
            p.material = mat(in.mat);
            for (int r = 0; r < 3; ++r) {
                for (int c = 0; c < 3; ++c) {
                    p.to_world.m[r][c] = in.to_world.m[r][c];
                    p.to_object.m[r][c] = in.to_object.m[r][c];
                }
                p.to_world.t[r] = in.to_world.t.e[r];
                p.to_object.t[r] = in.to_object.t.e[r];
            }
            instances.push_back(p);
        }
        lights.assign(world.lights.begin(), world.lights.end());
        std::memset(&desc, 0, sizeof(desc));
        desc.materials = materials.data();
        desc.n_materials = uint32_t(materials.size());
        desc.spheres = spheres.data();
        desc.n_spheres = uint32_t(spheres.size());
        desc.large_spheres = large.data();
        desc.n_large_spheres = uint32_t(large.size());
        desc.triangles = triangles.data();
        desc.n_triangles = uint32_t(triangles.size());
        desc.meshes = meshes.data();
        desc.n_meshes = uint32_t(meshes.size());
        desc.instances = instances.data();
        desc.n_instances = uint32_t(instances.size());
        desc.use_bvh = world.uses_bvh() ? 1 : 0;
        if (desc.use_bvh) {
            desc.flat_tree = tree(world.flat_tree());
            desc.instance_tree = tree(world.instances_tree());
        }
        desc.lights = lights.data();
        desc.n_lights = uint32_t(lights.size());
        desc.sky = world.sky ? 1 : 0;
        desc.sample_lights = world.sample_lights ? 1 : 0;
        desc.textures = textures.data();
        desc.n_textures = uint32_t(textures.size());
    }
};

// A geometry on the GPU. Holds the device scene; not copyable.
class gpu_scene {
public:
    gpu_scene() = default;
    gpu_scene(const gpu_scene&) = delete;
    gpu_scene& operator=(const gpu_scene&) = delete;
    ~gpu_scene() { pt_scene_destroy(scene_); }

    // Uploads a built geometry (geometry::build already called).
    pt_status upload(const geometry& world) {
        scene_arrays a;
        a.from(world);
        pt_scene_destroy(scene_);
        scene_ = nullptr;
        return pt_scene_create(&a.desc, &scene_);
    }

    // The whole frame as src/main.cpp lays it out: out is 3 * W * H floats,
    // top row first; aux is null or 7 * W * H floats (include/renderer.hpp:358-362).
    pt_status render(const camera& cam, int width, int height, int samples_per_pixel, int max_bounces, float* out,
                     uint64_t seed, int first_sample = 0, float* aux = nullptr, uint64_t* rays = nullptr,
                     int mode = PT_MODE_AUTO) const {
        const pt_camera c = camera_of(cam);
        pt_settings st;
        std::memset(&st, 0, sizeof(st));
        st.width = width;
        st.height = height;
        st.spp = samples_per_pixel;
        st.max_bounces = max_bounces;
        st.seed = seed;
        st.first_sample = first_sample;
        st.mode = mode;
        st.rng = PT_RNG_SAMPLE;
        return pt_render(scene_, &c, &st, out, aux, rays);
    }

    // One scanline: render_row_linear's signature and meaning.
    pt_status render_row_linear(const camera& cam, int j, int width, int height, int samples_per_pixel,
                                int max_bounces, float* out, uint64_t seed, int first_sample = 0,
                                float* aux = nullptr) const {
        const pt_camera c = camera_of(cam);
        return pt_render_row(scene_, &c, j, width, height, samples_per_pixel, max_bounces, out, seed, first_sample,
                             aux);
    }

    pt_scene* handle() const { return scene_; }

private:
    pt_scene* scene_ = nullptr;
};

}  // namespace photon_cuda
