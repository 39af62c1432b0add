// shim_check.cpp -- TEST INFRASTRUCTURE, not part of the product.
//
// Exercises include/photon_cuda_geometry.hpp the way a photon_tracer user
// would: builds the reference's own scenes with its build_world
// (include/renderer.hpp:335-343), uploads them through the bridge (which
// hands over the trees geometry::build made), then
//   * traces seeded rays on the GPU and compares t with geometry::hit's rec.t
//     ray by ray (bit for bit);
//   * renders a frame on the GPU and with render_row_linear on the CPU and
//     prints both image means.
// Prints one JSON line; exit code 0 when the hits agree. Built by
// oracle/build.py into oracle/_ref/shim_check (needs the reference checkout).
#include <cstdio>
#include <random>
#include <vector>

#include "renderer.hpp"
#include "../include/photon_cuda_geometry.hpp"

int main(int argc, char** argv) {
    const int id = argc > 1 ? std::atoi(argv[1]) : 3;  // scene_id: 0 materials, 1 field, 3 room
    const geometry world = build_world(static_cast<scene_id>(id), id != 0);
    const camera cam = make_camera(static_cast<scene_id>(id));
    photon_cuda::gpu_scene gpu;
    const pt_status up = gpu.upload(world);
    if (up != PT_OK) {
        std::printf("{\"upload\": %d, \"error\": \"%s\"}\n", up, pt_last_error());
        return up == PT_ERR_NO_DEVICE ? 3 : 2;
    }
    // Rays: origins near the camera, directions spread over the view.
    const size_t n = 100000;
    std::vector<float> rays(6 * n);
    std::mt19937_64 rng(5);
    auto u = [&rng] { return (rng() >> 11) * 0x1.0p-53; };
    for (size_t i = 0; i < n; ++i) {
        const ray r = cam.get_ray(float(u()), float(u()));
        for (int a = 0; a < 3; ++a) {
            rays[6 * i + a] = r.origin().e[a];
            rays[6 * i + 3 + a] = r.direction().e[a];
        }
    }
    std::vector<pt_hit> hits(n);
    if (pt_trace_closest(gpu.handle(), rays.data(), n, 0.001f, 1000.0f, hits.data()) != PT_OK) {
        std::printf("{\"trace\": \"%s\"}\n", pt_last_error());
        return 2;
    }
    size_t bad = 0, hit_count = 0;
    for (size_t i = 0; i < n; ++i) {
        const ray r(point3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]),
                    vec3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]));
        hit_record rec;
        const bool h = world.hit(r, 0.001f, 1000.0f, rec);
        hit_count += h;
        if (h != (hits[i].kind != PT_HIT_NONE) || (h && rec.t != hits[i].t)) ++bad;
    }
    const int W = 192, H = 108, spp = 64;
    std::vector<float> gpu_img(3 * W * H), cpu_img(3 * W * H);
    uint64_t rays_gpu = 0;
    if (gpu.render(cam, W, H, spp, 10, gpu_img.data(), 7, 0, nullptr, &rays_gpu) != PT_OK) {
        std::printf("{\"render\": \"%s\"}\n", pt_last_error());
        return 2;
    }
    rays_traced = 0;
    for (int j = 0; j < H; ++j)
        render_row_linear(world, cam, j, W, H, spp, 10, &cpu_img[3 * size_t(H - 1 - j) * W], 7, 0, nullptr);
    double mg = 0, mc = 0;
    for (size_t k = 0; k < cpu_img.size(); ++k) {
        mg += gpu_img[k];
        mc += cpu_img[k];
    }
    std::printf("{\"scene\": %d, \"rays\": %zu, \"hits\": %zu, \"hit_mismatch\": %zu, \"gpu_mean\": %.6f, "
                "\"cpu_mean\": %.6f, \"gpu_rays\": %llu, \"cpu_rays\": %lld}\n",
                id, n, hit_count, bad, mg / cpu_img.size(), mc / cpu_img.size(), (unsigned long long)rays_gpu,
                (long long)rays_traced);
    return bad == 0 ? 0 : 1;
}
