// Procedural scenes, cameras and ray sets.
//
// Two families:
//  * the reference's own scenes (materials, field, room), rebuilt value for
//    value so renders can be checked against the reference's statistical
//    fixtures (tests/reference.json of photon_tracer). Their constants and the
//    order of random draws follow include/renderer.hpp:158-208 and 245-268;
//  * the benchmark workloads: random spheres (400x225), a closed room with a
//    displaced icosphere (1024x1024), 10,000 instances of three procedural
//    meshes (1920x1080), and the scenes of the 64-scene batch. These have no
//    counterpart in the reference; they draw every number in a fixed order
//    from std::mt19937(seed) as rng() * 2^-32, the reference's convention
//    (include/renderer.hpp:179-180), so every consumer gets identical arrays.
#include "pt_host.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <random>
#include <utility>
#include <vector>

struct pt_generated {
    std::vector<pt_material> materials;
    std::vector<pt_sphere> spheres, large;
    std::vector<pt_triangle> triangles;
    std::vector<std::vector<pt_triangle>> mesh_tris;
    std::vector<pt_mesh> meshes;
    std::vector<pt_instance> instances;
    std::vector<std::vector<uint8_t>> images;  // sRGB bytes of the textures
    std::vector<pt_texture> textures;
    pt_scene_desc desc;
    pt_camera cam;
};

namespace pt {

pt_triangle make_triangle(V3 a, V3 b, V3 c, V3 na, V3 nb, V3 nc, uint32_t material) {
    pt_triangle t;
    std::memset(&t, 0, sizeof(t));
    const V3 e1 = b - a, e2 = c - a;
    store(t.p0, a);
    store(t.e1, e1);
    store(t.e2, e2);
    store(t.n0, na);
    store(t.n1, nb);
    store(t.n2, nc);
    store(t.face_normal, normalize(cross(e1, e2)));
    store(t.p1, b);
    store(t.p2, c);
    t.material = material;
    return t;
}

pt_triangle make_triangle(V3 a, V3 b, V3 c, uint32_t material) {
    pt_triangle t = make_triangle(a, b, c, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, material);
    std::memcpy(t.n0, t.face_normal, sizeof(t.n0));
    std::memcpy(t.n1, t.face_normal, sizeof(t.n1));
    std::memcpy(t.n2, t.face_normal, sizeof(t.n2));
    return t;
}

}  // namespace pt

using namespace pt;

namespace {

// ---- small builders -------------------------------------------------------------
struct SceneBuilder {
    pt_generated* g;
    uint32_t material(uint32_t type, V3 albedo, V3 emission, float fuzz, float ior) {
        pt_material m;
        m.type = type;
        store(m.albedo, albedo);
        store(m.emission, emission);
        m.fuzz = fuzz;
        m.ior = ior;
        m.texture = 0;
        g->materials.push_back(m);
        return static_cast<uint32_t>(g->materials.size() - 1);
    }
    uint32_t lambertian(V3 a) { return material(PT_MAT_LAMBERTIAN, a, V3{0, 0, 0}, 0, 1.5f); }
    uint32_t textured(V3 a, uint32_t texture) {
        const uint32_t m = lambertian(a);
        g->materials[m].texture = texture;
        return m;
    }
    // A texture of w x h sRGB texels; returns its 1-based number for materials.
    uint32_t texture(int w, int h, std::vector<uint8_t> rgb) {
        g->images.push_back(std::move(rgb));
        g->textures.push_back({w, h, nullptr});
        return uint32_t(g->textures.size());
    }
    // metal(a, f): fuzz(f < 1 ? f : 1) (include/material.hpp:83)
    uint32_t metal(V3 a, float f) { return material(PT_MAT_METAL, a, V3{0, 0, 0}, f < 1 ? f : 1, 1.5f); }
    uint32_t dielectric(float ior) { return material(PT_MAT_DIELECTRIC, V3{0, 0, 0}, V3{0, 0, 0}, 0, ior); }
    uint32_t light(V3 e) { return material(PT_MAT_DIFFUSE_LIGHT, V3{0, 0, 0}, e, 0, 1.5f); }
    void sphere(V3 c, float r, uint32_t m) { g->spheres.push_back({{c.x, c.y, c.z}, r, m}); }
    void large_sphere(V3 c, float r, uint32_t m) { g->large.push_back({{c.x, c.y, c.z}, r, m}); }
    // add_quad (include/renderer.hpp:235-238): (p, p+e1, p+e1+e2), (p, p+e1+e2, p+e2)
    void quad(V3 p, V3 e1, V3 e2, uint32_t m) {
        g->triangles.push_back(make_triangle(p, p + e1, p + e1 + e2, m));
        g->triangles.push_back(make_triangle(p, p + e1 + e2, p + e2, m));
    }
};

V3 p3(double x, double y, double z) { return V3{float(x), float(y), float(z)}; }

// ---- the reference's scenes -----------------------------------------------------------
void ref_materials_scene(SceneBuilder& b, bool field) {
    const uint32_t ground = b.lambertian(p3(0.8, 0.8, 0.0));
    const uint32_t matte = b.lambertian(p3(0.1, 0.2, 0.5));
    const uint32_t glass = b.dielectric(1.5f);
    const uint32_t gold = b.metal(p3(0.8, 0.6, 0.2), float(0.1));
    b.large_sphere(p3(0, -100.5, -1), 100.0f, ground);
    b.sphere(p3(0, 0.0, -1), 0.5f, matte);
    b.sphere(p3(-1, 0.0, -1), 0.5f, glass);
    b.sphere(p3(-1, 0.0, -1), -0.4f, glass);
    b.sphere(p3(1, 0.0, -1), 0.5f, gold);
    if (!field) return;
    std::mt19937 rng(7);
    auto u = [&rng] { return rng() * 0x1.0p-32; };
    for (int a = -15; a < 15; ++a) {
        for (int bb = -15; bb < -1; ++bb) {
            const double jitter_x = u();
            const double jitter_z = u();
            const V3 c = p3(a * 0.2 + 0.12 * jitter_x, -0.44, bb * 0.2 + 0.12 * jitter_z);
            // clamp(std::round(c.x()), -1.0, 1.0) in float
            float rx = std::round(c.x);
            rx = rx < -1.0f ? -1.0f : rx > 1.0f ? 1.0f : rx;
            const V3 d = c - V3{rx, float(-0.44), float(-1)};
            if (double(dot(d, d)) < 0.36) continue;
            const double pick = u();
            uint32_t m;
            if (pick < 0.7) {
                double albedo[3];
                for (double& x : albedo) { x = u(); x *= u(); }
                m = b.lambertian(p3(albedo[0], albedo[1], albedo[2]));
            } else if (pick < 0.9) {
                double albedo[3];
                for (double& x : albedo) x = 0.5 + 0.5 * u();
                const double fuzz = 0.3 * u();
                m = b.metal(p3(albedo[0], albedo[1], albedo[2]), float(fuzz));
            } else {
                m = glass;
            }
            b.sphere(c, 0.06f, m);
        }
    }
}

void ref_room_scene(SceneBuilder& b) {
    b.g->desc.sky = 0;
    const uint32_t white = b.lambertian(p3(0.73, 0.73, 0.73));
    const uint32_t red = b.lambertian(p3(0.65, 0.05, 0.05));
    const uint32_t green = b.lambertian(p3(0.12, 0.45, 0.15));
    const uint32_t lamp = b.light(p3(30, 27, 22));
    const double x0 = -1.75, x1 = 1.75, y0 = -1, y1 = 1, z0 = -3.5, z1 = 0.5;
    b.quad(p3(x0, y0, z1), p3(x1 - x0, 0, 0), p3(0, 0, z0 - z1), white);  // floor
    b.quad(p3(x0, y1, z1), p3(x1 - x0, 0, 0), p3(0, 0, z0 - z1), white);  // ceiling
    b.quad(p3(x0, y0, z0), p3(x1 - x0, 0, 0), p3(0, y1 - y0, 0), white);  // back
    b.quad(p3(x0, y0, z1), p3(x1 - x0, 0, 0), p3(0, y1 - y0, 0), white);  // front
    b.quad(p3(x0, y0, z1), p3(0, 0, z0 - z1), p3(0, y1 - y0, 0), red);    // left
    b.quad(p3(x1, y0, z1), p3(0, 0, z0 - z1), p3(0, y1 - y0, 0), green);  // right
    b.sphere(p3(0, 0.72, -2.0), 0.14f, lamp);
    b.sphere(p3(-0.8, -0.55, -2.3), 0.45f, b.dielectric(1.5f));
    b.sphere(p3(0.85, -0.6, -1.8), 0.4f, b.metal(p3(0.9, 0.9, 0.9), float(0.02)));
    b.sphere(p3(0.15, -0.75, -2.9), 0.25f, b.lambertian(p3(0.1, 0.2, 0.5)));
}

// ---- noise ------------------------------------------------------------------------------
uint32_t hash32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Lattice value in [-1, 1] at integer point (i, j, k) for seed.
double lattice(int i, int j, int k, uint32_t seed) {
    uint32_t h = hash32(seed ^ 0x9e3779b9u);
    h = hash32(h ^ uint32_t(i) * 0x8da6b343u);
    h = hash32(h ^ uint32_t(j) * 0xd8163841u);
    h = hash32(h ^ uint32_t(k) * 0xcb1ab31fu);
    return (h >> 8) * (2.0 / 16777216.0) - 1.0;
}

// Trilinear value noise with smoothstep weights.
double value_noise(double x, double y, double z, uint32_t seed) {
    const double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    const int ix = int(fx), iy = int(fy), iz = int(fz);
    auto s = [](double t) { return t * t * (3 - 2 * t); };
    const double tx = s(x - fx), ty = s(y - fy), tz = s(z - fz);
    double acc = 0;
    for (int c = 0; c < 8; ++c) {
        const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
        const double w = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
        acc += w * lattice(ix + dx, iy + dy, iz + dz, seed);
    }
    return acc;
}

// Sum of `octaves` octaves: frequency doubling from f0, amplitude halving from 1.
double fbm(double x, double y, double z, uint32_t seed, int octaves, double f0) {
    double sum = 0, amp = 1, f = f0;
    for (int o = 0; o < octaves; ++o) {
        sum += amp * value_noise(x * f, y * f, z * f, seed + 101u * uint32_t(o));
        amp *= 0.5;
        f *= 2;
    }
    return sum;
}

// ---- meshes ----------------------------------------------------------------------------
struct Mesh {
    std::vector<std::array<double, 3>> v;
    std::vector<std::array<uint32_t, 3>> f;
};

Mesh icosphere(int subdivisions) {
    Mesh m;
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    const double base[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                                {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& p : base) {
        const double l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        m.v.push_back({p[0] / l, p[1] / l, p[2] / l});
    }
    m.f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
           {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
           {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (int s = 0; s < subdivisions; ++s) {
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> mid;
        auto midpoint = [&](uint32_t a, uint32_t b) {
            const auto key = std::make_pair(std::min(a, b), std::max(a, b));
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            double p[3];
            for (int k = 0; k < 3; ++k) p[k] = 0.5 * (m.v[a][k] + m.v[b][k]);
            const double l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
            m.v.push_back({p[0] / l, p[1] / l, p[2] / l});
            const uint32_t idx = uint32_t(m.v.size() - 1);
            mid.emplace(key, idx);
            return idx;
        };
        std::vector<std::array<uint32_t, 3>> next;
        next.reserve(m.f.size() * 4);
        for (const auto& f : m.f) {
            const uint32_t a = midpoint(f[0], f[1]), b = midpoint(f[1], f[2]), c = midpoint(f[2], f[0]);
            next.push_back({f[0], a, c});
            next.push_back({f[1], b, a});
            next.push_back({f[2], c, b});
            next.push_back({a, b, c});
        }
        m.f.swap(next);
    }
    return m;
}

// Triangles with area-weighted vertex normals: each face adds cross(b - a, c - a)
// (twice its area times its normal) to its corners, as include/obj.hpp:198-204 does.
std::vector<pt_triangle> smooth_triangles(const Mesh& m, uint32_t material) {
    std::vector<V3> pos(m.v.size());
    for (size_t i = 0; i < m.v.size(); ++i) pos[i] = p3(m.v[i][0], m.v[i][1], m.v[i][2]);
    std::vector<V3> acc(m.v.size(), V3{0, 0, 0});
    for (const auto& f : m.f) {
        const V3 n = cross(pos[f[1]] - pos[f[0]], pos[f[2]] - pos[f[0]]);
        for (int k = 0; k < 3; ++k) acc[f[k]] = acc[f[k]] + n;
    }
    std::vector<pt_triangle> out;
    out.reserve(m.f.size());
    for (const auto& f : m.f)
        out.push_back(make_triangle(pos[f[0]], pos[f[1]], pos[f[2]], normalize(acc[f[0]]), normalize(acc[f[1]]),
                                    normalize(acc[f[2]]), material));
    return out;
}

// Displaces an icosphere radially: radius * (1 + amp * fbm4(direction)), then
// moves it to center.
void displace(Mesh& m, double radius, double amp, uint32_t seed, const double center[3]) {
    for (auto& p : m.v) {
        const double n = fbm(p[0], p[1], p[2], seed, 4, 2.0);
        const double r = radius * (1.0 + amp * n);
        for (int k = 0; k < 3; ++k) p[k] = center[k] + r * p[k];
    }
}

// (p, q) torus knot tube: `along` rings of `around` vertices, two triangles
// per quad, normals the tube's outward direction.
std::vector<pt_triangle> torus_knot(int p, int q, double tube, int along, int around, uint32_t material) {
    const double R = 1.0, r = 0.45;
    auto curve = [&](double phi, double out[3]) {
        const double rr = R + r * std::cos(q * phi);
        out[0] = rr * std::cos(p * phi);
        out[1] = r * std::sin(q * phi);
        out[2] = rr * std::sin(p * phi);
    };
    const double two_pi = 2 * M_PI;
    std::vector<V3> pos(size_t(along) * around), nrm(size_t(along) * around);
    for (int i = 0; i < along; ++i) {
        const double phi = two_pi * i / along, h = 1e-4;
        double c[3], a[3], b[3];
        curve(phi, c);
        curve(phi + h, a);
        curve(phi - h, b);
        double T[3], A[3];
        for (int k = 0; k < 3; ++k) {
            T[k] = a[k] - b[k];
            A[k] = a[k] - 2 * c[k] + b[k];
        }
        auto norm = [](double v[3]) {
            const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            for (int k = 0; k < 3; ++k) v[k] /= l;
        };
        norm(T);
        const double ta = T[0] * A[0] + T[1] * A[1] + T[2] * A[2];
        double N[3] = {A[0] - ta * T[0], A[1] - ta * T[1], A[2] - ta * T[2]};
        norm(N);
        double B[3] = {T[1] * N[2] - T[2] * N[1], T[2] * N[0] - T[0] * N[2], T[0] * N[1] - T[1] * N[0]};
        for (int j = 0; j < around; ++j) {
            const double th = two_pi * j / around, cs = std::cos(th), sn = std::sin(th);
            double d[3];
            for (int k = 0; k < 3; ++k) d[k] = cs * N[k] + sn * B[k];
            pos[size_t(i) * around + j] = p3(c[0] + tube * d[0], c[1] + tube * d[1], c[2] + tube * d[2]);
            nrm[size_t(i) * around + j] = p3(d[0], d[1], d[2]);
        }
    }
    std::vector<pt_triangle> out;
    out.reserve(size_t(2) * along * around);
    for (int i = 0; i < along; ++i)
        for (int j = 0; j < around; ++j) {
            const size_t a = size_t(i) * around + j, b = size_t((i + 1) % along) * around + j,
                         c = size_t((i + 1) % along) * around + (j + 1) % around,
                         d = size_t(i) * around + (j + 1) % around;
            // Wound so the face normal points out of the tube, like the vertex normals.
            out.push_back(make_triangle(pos[a], pos[c], pos[b], nrm[a], nrm[c], nrm[b], material));
            out.push_back(make_triangle(pos[a], pos[d], pos[c], nrm[a], nrm[d], nrm[c], material));
        }
    return out;
}

// A cells x cells grid over [-1, 1]^2 in x and z, height amp * fbm5.
std::vector<pt_triangle> heightfield(int cells, double amp, uint32_t seed, uint32_t material) {
    Mesh m;
    const int n = cells + 1;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const double x = -1 + 2.0 * j / cells, z = -1 + 2.0 * i / cells;
            m.v.push_back({x, amp * fbm(x, 0.37, z, seed, 5, 1.5), z});
        }
    for (int i = 0; i < cells; ++i)
        for (int j = 0; j < cells; ++j) {
            const uint32_t a = uint32_t(i * n + j), b = uint32_t(i * n + j + 1), c = uint32_t((i + 1) * n + j + 1),
                           d = uint32_t((i + 1) * n + j);
            m.f.push_back({a, c, b});
            m.f.push_back({a, d, c});
        }
    return smooth_triangles(m, material);
}

// ---- benchmark scenes ---------------------------------------------------------------------
// Random spheres: large ground r=1000, a 22x22 grid of r=0.2 spheres (or n
// spheres scattered over the same area), three r=1 spheres, one light r=2.
void random_spheres_scene(SceneBuilder& b, uint64_t seed, int n_small) {
    std::mt19937 rng(static_cast<uint32_t>(seed));
    auto u = [&rng] { return rng() * 0x1.0p-32; };
    b.large_sphere(p3(0, -1000, 0), 1000.0f, b.lambertian(p3(0.5, 0.5, 0.5)));
    const uint32_t glass = b.dielectric(1.5f);
    auto small = [&](double cx, double cz) {
        const double pick = u();
        uint32_t m;
        if (pick < 0.8) {
            double albedo[3];
            for (double& x : albedo) { x = u(); x *= u(); }
            m = b.lambertian(p3(albedo[0], albedo[1], albedo[2]));
        } else if (pick < 0.95) {
            double albedo[3];
            for (double& x : albedo) x = 0.5 + 0.5 * u();
            const double fuzz = 0.5 * u();
            m = b.metal(p3(albedo[0], albedo[1], albedo[2]), float(fuzz));
        } else {
            m = glass;
        }
        b.sphere(p3(cx, 0.2, cz), 0.2f, m);
    };
    if (n_small <= 0) {
        for (int a = -11; a < 11; ++a)
            for (int bb = -11; bb < 11; ++bb) {
                const double ux = u();
                const double uz = u();
                small(a + 0.9 * ux, bb + 0.9 * uz);
            }
    } else {
        for (int k = 0; k < n_small; ++k) {
            const double ux = u();
            const double uz = u();
            small(-11 + 22 * ux, -11 + 22 * uz);
        }
    }
    b.sphere(p3(0, 1, 0), 1.0f, glass);
    b.sphere(p3(-4, 1, 0), 1.0f, b.lambertian(p3(0.4, 0.2, 0.1)));
    b.sphere(p3(4, 1, 0), 1.0f, b.metal(p3(0.7, 0.6, 0.5), 0.0f));
    b.sphere(p3(0, 10, 0), 2.0f, b.light(p3(4, 4, 4)));
}

// Closed room [-1,1]^3 without a front wall, ceiling light, glass sphere and a
// displaced icosphere of `subdiv` subdivisions (6: 81,920 triangles).
void room_mesh_scene(SceneBuilder& b, uint64_t seed, int subdiv) {
    b.g->desc.sky = 0;
    const uint32_t white = b.lambertian(p3(0.73, 0.73, 0.73));
    const uint32_t red = b.lambertian(p3(0.65, 0.05, 0.05));
    const uint32_t green = b.lambertian(p3(0.12, 0.45, 0.15));
    b.quad(p3(-1, -1, 1), p3(2, 0, 0), p3(0, 0, -2), white);  // floor
    b.quad(p3(-1, 1, 1), p3(2, 0, 0), p3(0, 0, -2), white);   // ceiling
    b.quad(p3(-1, -1, -1), p3(2, 0, 0), p3(0, 2, 0), white);  // back
    b.quad(p3(-1, -1, 1), p3(0, 0, -2), p3(0, 2, 0), red);    // left
    b.quad(p3(1, -1, 1), p3(0, 0, -2), p3(0, 2, 0), green);   // right
    b.sphere(p3(0, 0.82, -0.1), 0.15f, b.light(p3(15, 15, 15)));
    b.sphere(p3(0.5, -0.8, 0.35), 0.2f, b.dielectric(1.5f));
    Mesh ico = icosphere(subdiv);
    const double center[3] = {-0.2, -0.5, -0.25};
    displace(ico, 0.45, 0.05 / 0.45, static_cast<uint32_t>(seed), center);
    const std::vector<pt_triangle> tris = smooth_triangles(ico, b.lambertian(p3(0.8, 0.8, 0.8)));
    b.g->triangles.insert(b.g->triangles.end(), tris.begin(), tris.end());
}

// The reference's room lit by emissive meshes instead of its lamp sphere (no
// counterpart in the reference, whose light sampling covers spheres only,
// README.md:453-456): a lamp of 80 emissive triangles (a once-subdivided
// icosphere, flat-shaded, faces outward) where the sphere lamp hangs, an
// emissive ceiling panel (2 triangles facing down) and a small light sphere,
// over glass, rough metal (fuzz 0.25), a mirror (fuzz 0) and matte spheres:
// the scene of the extended light-sampling tests.
void mesh_light_room_scene(SceneBuilder& b) {
    b.g->desc.sky = 0;
    const uint32_t white = b.lambertian(p3(0.73, 0.73, 0.73));
    const uint32_t red = b.lambertian(p3(0.65, 0.05, 0.05));
    const uint32_t green = b.lambertian(p3(0.12, 0.45, 0.15));
    const double x0 = -1.75, x1 = 1.75, y0 = -1, y1 = 1, z0 = -3.5, z1 = 0.5;
    b.quad(p3(x0, y0, z1), p3(x1 - x0, 0, 0), p3(0, 0, z0 - z1), white);  // floor
    b.quad(p3(x0, y1, z1), p3(x1 - x0, 0, 0), p3(0, 0, z0 - z1), white);  // ceiling
    b.quad(p3(x0, y0, z0), p3(x1 - x0, 0, 0), p3(0, y1 - y0, 0), white);  // back
    b.quad(p3(x0, y0, z1), p3(x1 - x0, 0, 0), p3(0, y1 - y0, 0), white);  // front
    b.quad(p3(x0, y0, z1), p3(0, 0, z0 - z1), p3(0, y1 - y0, 0), red);    // left
    b.quad(p3(x1, y0, z1), p3(0, 0, z0 - z1), p3(0, y1 - y0, 0), green);  // right
    const uint32_t lamp = b.light(p3(30, 27, 22));
    const Mesh ico = icosphere(1);
    const double lc[3] = {0, 0.72, -2.0}, lr = 0.14;
    for (const auto& f : ico.f) {
        V3 c[3];
        for (int k = 0; k < 3; ++k)
            c[k] = p3(lc[0] + lr * ico.v[f[k]][0], lc[1] + lr * ico.v[f[k]][1], lc[2] + lr * ico.v[f[k]][2]);
        b.g->triangles.push_back(make_triangle(c[0], c[1], c[2], lamp));
    }
    b.quad(p3(-0.3, 0.999, -1.2), p3(0, 0, -0.6), p3(0.6, 0, 0), b.light(p3(3, 3, 3)));  // panel, facing down
    b.sphere(p3(0.9, 0.5, -2.6), 0.05f, b.light(p3(40, 40, 40)));
    b.sphere(p3(-0.8, -0.55, -2.3), 0.45f, b.dielectric(1.5f));
    b.sphere(p3(0.85, -0.6, -1.8), 0.4f, b.metal(p3(0.9, 0.8, 0.7), 0.25f));
    b.sphere(p3(0.3, -0.8, -1.3), 0.2f, b.metal(p3(0.9, 0.9, 0.9), 0.0f));
    b.sphere(p3(0.15, -0.75, -2.9), 0.25f, b.lambertian(p3(0.1, 0.2, 0.5)));
}

// 10,000 instances of a displaced icosphere (20,480), a (3,7) torus knot
// (50,000) and a 256x256 heightfield (131,072) over a 200x200 area, ground
// sphere r=1000, 8 light spheres r=3 emission 8 at height 40.
void instances_scene(SceneBuilder& b, uint64_t seed, int n_instances) {
    pt_generated* g = b.g;
    std::mt19937 rng(static_cast<uint32_t>(seed));
    auto u = [&rng] { return rng() * 0x1.0p-32; };
    b.large_sphere(p3(0, -1000, 0), 1000.0f, b.lambertian(p3(0.5, 0.5, 0.5)));
    for (int k = 0; k < 8; ++k)
        b.sphere(p3(-75 + 50 * (k % 4), 40, -40 + 80 * (k / 4)), 3.0f, b.light(p3(8, 8, 8)));

    Mesh ico = icosphere(5);
    const double zero[3] = {0, 0, 0};
    displace(ico, 1.0, 0.08, static_cast<uint32_t>(seed) + 17u, zero);
    g->mesh_tris.push_back(smooth_triangles(ico, b.lambertian(p3(0.8, 0.3, 0.3))));
    g->mesh_tris.push_back(torus_knot(3, 7, 0.15, 1000, 25, b.metal(p3(0.9, 0.8, 0.5), 0.1f)));
    g->mesh_tris.push_back(heightfield(256, 0.3, static_cast<uint32_t>(seed) + 29u, b.lambertian(p3(0.3, 0.6, 0.3))));

    const uint32_t glass = b.dielectric(1.5f);
    for (int k = 0; k < n_instances; ++k) {
        const double u1 = u(), u2 = u(), u3 = u();
        const double ls = u(), tx = u(), tz = u(), which = u(), over = u();
        // Uniform rotation from three uniforms (Shoemake): quaternion (x, y, z, w).
        const double s1 = std::sqrt(1 - u1), s2 = std::sqrt(u1);
        const double qx = s1 * std::sin(2 * M_PI * u2), qy = s1 * std::cos(2 * M_PI * u2);
        const double qz = s2 * std::sin(2 * M_PI * u3), qw = s2 * std::cos(2 * M_PI * u3);
        const double R[3][3] = {{1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qz * qw), 2 * (qx * qz + qy * qw)},
                                {2 * (qx * qy + qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qx * qw)},
                                {2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)}};
        const double scale = 0.5 * std::pow(4.0, ls);  // log-uniform in [0.5, 2]
        pt_affine w;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) w.m[i][j] = float(R[i][j] * scale);
        w.t[0] = float(-100 + 200 * tx);
        w.t[1] = float(scale);
        w.t[2] = float(-100 + 200 * tz);
        uint32_t mat = PT_NO_MATERIAL;
        if (over < 0.05) {
            const double c0 = u(), c1 = u(), c2 = u(), kind = u();
            if (kind < 0.6) mat = b.lambertian(p3(c0, c1, c2));
            else if (kind < 0.9) mat = b.metal(p3(0.5 + 0.5 * c0, 0.5 + 0.5 * c1, 0.5 + 0.5 * c2), float(0.3 * kind));
            else mat = glass;
        }
        pt_instance in;
        in.mesh = which < 1.0 / 3 ? 0u : which < 2.0 / 3 ? 1u : 2u;
        in.material = mat;
        in.to_world = w;
        in.to_object = affine_inverse(w);
        g->instances.push_back(in);
    }
}

// A textured scene (no counterpart among the reference's scenes; it exercises
// lambertian::texture, include/material.hpp:50-72): the reference's room
// with seeded sRGB checker textures on the floor and the back wall, a
// textured sphere (texture coordinates (0, 0), as sphere::fill leaves them),
// and six instances of an icosphere with longitude/latitude coordinates,
// every other one with a textured override material.
void textured_scene(SceneBuilder& b, uint64_t seed) {
    pt_generated* g = b.g;
    std::mt19937 rng(static_cast<uint32_t>(seed));
    auto u = [&rng] { return rng() * 0x1.0p-32; };
    auto checker = [&](int w, int h, int cells) {
        std::vector<uint8_t> rgb(3 * size_t(w) * h);
        std::vector<uint8_t> cell(3 * cells * cells);
        for (auto& c : cell) c = uint8_t(40 + 215 * u());
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x)
                for (int c = 0; c < 3; ++c) {
                    const int cx = x * cells / w, cy = y * cells / h;
                    rgb[3 * (size_t(y) * w + x) + c] = uint8_t((cell[3 * (cy * cells + cx) + c] + 7 * ((x + y) & 7)) & 255);
                }
        return rgb;
    };
    const uint32_t floor_tex = b.texture(96, 64, checker(96, 64, 8));
    const uint32_t wall_tex = b.texture(37, 53, checker(37, 53, 5));
    g->desc.sky = 0;
    const uint32_t white = b.lambertian(p3(0.73, 0.73, 0.73));
    const uint32_t red = b.lambertian(p3(0.65, 0.05, 0.05));
    const uint32_t green = b.lambertian(p3(0.12, 0.45, 0.15));
    const uint32_t floor_mat = b.textured(p3(0.9, 0.9, 0.9), floor_tex);
    const uint32_t wall_mat = b.textured(p3(0.8, 0.8, 0.8), wall_tex);
    const double x0 = -1.75, x1 = 1.75, y0 = -1, y1 = 1, z0 = -3.5, z1 = 0.5;
    // a quad with texture coordinates (0,0) (r,0) (r,r) (0,r) at p, p+e1, p+e1+e2, p+e2
    auto tquad = [&](V3 p, V3 e1, V3 e2, uint32_t m, float r) {
        pt_triangle a = make_triangle(p, p + e1, p + e1 + e2, m), c = make_triangle(p, p + e1 + e2, p + e2, m);
        const float ua[6] = {0, 0, r, 0, r, r}, uc[6] = {0, 0, r, r, 0, r};
        std::memcpy(a.uv, ua, sizeof(ua));
        std::memcpy(c.uv, uc, sizeof(uc));
        g->triangles.push_back(a);
        g->triangles.push_back(c);
    };
    tquad(p3(x0, y0, z1), p3(x1 - x0, 0, 0), p3(0, 0, z0 - z1), floor_mat, 2.5f);  // floor, repeating
    b.quad(p3(x0, y1, z1), p3(x1 - x0, 0, 0), p3(0, 0, z0 - z1), white);          // ceiling
    tquad(p3(x0, y0, z0), p3(x1 - x0, 0, 0), p3(0, y1 - y0, 0), wall_mat, 1.0f);  // back
    b.quad(p3(x0, y0, z1), p3(x1 - x0, 0, 0), p3(0, y1 - y0, 0), white);          // front
    b.quad(p3(x0, y0, z1), p3(0, 0, z0 - z1), p3(0, y1 - y0, 0), red);            // left
    b.quad(p3(x1, y0, z1), p3(0, 0, z0 - z1), p3(0, y1 - y0, 0), green);          // right
    b.sphere(p3(0, 0.72, -2.0), 0.14f, b.light(p3(30, 27, 22)));
    b.sphere(p3(0.15, -0.75, -2.9), 0.25f, b.textured(p3(1, 1, 1), wall_tex));

    Mesh ico = icosphere(3);
    std::vector<pt_triangle> tris = smooth_triangles(ico, b.textured(p3(0.95, 0.95, 0.95), floor_tex));
    for (size_t f = 0; f < ico.f.size(); ++f)
        for (int k = 0; k < 3; ++k) {
            const auto& v = ico.v[ico.f[f][k]];
            tris[f].uv[2 * k] = float(std::atan2(v[2], v[0]) / (2 * M_PI) + 0.5);
            tris[f].uv[2 * k + 1] = float(std::asin(std::max(-1.0, std::min(1.0, v[1]))) / M_PI + 0.5);
        }
    g->mesh_tris.push_back(tris);
    for (int k = 0; k < 6; ++k) {
        const double s = 0.18 + 0.1 * u(), yaw = 2 * M_PI * u();
        pt_affine w;
        std::memset(&w, 0, sizeof(w));
        const double c = std::cos(yaw), sn = std::sin(yaw);
        const double R[3][3] = {{c, 0, sn}, {0, 1, 0}, {-sn, 0, c}};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) w.m[i][j] = float(R[i][j] * s);
        w.t[0] = float(-1.2 + 0.5 * k);
        w.t[1] = float(-1 + s);
        w.t[2] = float(-1.6 - 0.25 * (k % 3));
        pt_instance in;
        in.mesh = 0;
        in.material = (k % 2) ? b.textured(p3(0.7 + 0.3 * u(), 0.7, 0.7), wall_tex) : PT_NO_MATERIAL;
        in.to_world = w;
        in.to_object = affine_inverse(w);
        g->instances.push_back(in);
    }
}

void finish(pt_generated* g) {
    pt_scene_desc& d = g->desc;
    for (size_t k = 0; k < g->textures.size(); ++k) g->textures[k].rgb = g->images[k].data();
    d.textures = g->textures.data();
    d.n_textures = uint32_t(g->textures.size());
    g->meshes.clear();
    for (auto& t : g->mesh_tris) {
        pt_mesh m;
        std::memset(&m, 0, sizeof(m));
        m.triangles = t.data();
        m.n_triangles = uint32_t(t.size());
        g->meshes.push_back(m);
    }
    d.materials = g->materials.data();
    d.n_materials = uint32_t(g->materials.size());
    d.spheres = g->spheres.data();
    d.n_spheres = uint32_t(g->spheres.size());
    d.large_spheres = g->large.data();
    d.n_large_spheres = uint32_t(g->large.size());
    d.triangles = g->triangles.data();
    d.n_triangles = uint32_t(g->triangles.size());
    d.meshes = g->meshes.data();
    d.n_meshes = uint32_t(g->meshes.size());
    d.instances = g->instances.data();
    d.n_instances = uint32_t(g->instances.size());
}

}  // namespace

extern "C" {

pt_status pt_camera_look_at(const float lookfrom[3], const float lookat[3], double vfov_deg, double aspect,
                            pt_camera* out) {
    if (!lookfrom || !lookat || !out) return fail(PT_ERR_INVALID_ARG, "pt_camera_look_at: null pointer");
    // include/camera.hpp:18-34, the aspect ratio a parameter.
    const double viewport_height = 2.0 * std::tan(vfov_deg * M_PI / 360.0);
    const double viewport_width = aspect * viewport_height;
    const V3 from = load(lookfrom), at = load(lookat);
    const V3 w = normalize(from - at);
    const V3 u = normalize(cross(V3{0, 1, 0}, w));
    const V3 v = cross(w, u);
    const V3 horizontal = u * float(viewport_width);
    const V3 vertical = v * float(viewport_height);
    const V3 llc = from - horizontal * 0.5f - vertical * 0.5f - w;
    store(out->origin, from);
    store(out->lower_left, llc);
    store(out->horizontal, horizontal);
    store(out->vertical, vertical);
    return PT_OK;
}

pt_status pt_generate(pt_gen_params* params, pt_generated** out) {
    clear_error();
    if (!params || !out) return fail(PT_ERR_INVALID_ARG, "pt_generate: null pointer");
    *out = nullptr;
    std::unique_ptr<pt_generated> g(new pt_generated());
    std::memset(&g->desc, 0, sizeof(g->desc));
    g->desc.sky = 1;
    g->desc.sample_lights = 1;
    SceneBuilder b{g.get()};
    int use_bvh_default = 1;
    double aspect = 16.0 / 9.0;
    float from[3], at[3];
    double vfov = 90;
    int width = 0, height = 0, spp = 0;
    switch (params->kind) {
        case PT_GEN_REF_MATERIALS:
        case PT_GEN_REF_FIELD: {
            const bool field = params->kind == PT_GEN_REF_FIELD;
            ref_materials_scene(b, field);
            use_bvh_default = field ? 1 : 0;  // src/main.cpp:66
            // make_camera (include/renderer.hpp:212-218)
            if (field) {
                store(from, p3(0, 1.0, 1.2)); store(at, p3(0, -0.3, -1.2)); vfov = 55.0;
            } else {
                store(from, p3(0, 0, 0)); store(at, p3(0, 0, -1)); vfov = 90.0;
            }
            width = 960; height = 540; spp = 200;
            break;
        }
        case PT_GEN_REF_ROOM:
            ref_room_scene(b);
            store(from, p3(0, 0, 0.3)); store(at, p3(0, -0.15, -3.0)); vfov = 62.0;
            width = 960; height = 540; spp = 200;
            break;
        case PT_GEN_RANDOM_SPHERES:
            random_spheres_scene(b, params->seed, params->param);
            store(from, p3(13, 2, 3)); store(at, p3(0, 0, 0)); vfov = 20.0;
            width = 400; height = 225; spp = 16;
            break;
        case PT_GEN_ROOM_MESH:
            room_mesh_scene(b, params->seed, params->param > 0 ? params->param : 6);
            store(from, p3(0, 0, 3.3)); store(at, p3(0, 0, 0)); vfov = 40.0;
            aspect = 1.0;
            width = 1024; height = 1024; spp = 64;
            break;
        case PT_GEN_INSTANCES:
            instances_scene(b, params->seed, params->param > 0 ? params->param : 10000);
            store(from, p3(0, 35, 140)); store(at, p3(0, 0, 0)); vfov = 45.0;
            width = 1920; height = 1080; spp = 32;
            break;
        case PT_GEN_MESH_LIGHT:
            mesh_light_room_scene(b);
            store(from, p3(0, 0, 0.3)); store(at, p3(0, -0.15, -3.0)); vfov = 62.0;
            width = 960; height = 540; spp = 200;
            break;
        case PT_GEN_TEXTURED:
            textured_scene(b, params->seed);
            store(from, p3(0, 0, 0.3)); store(at, p3(0, -0.15, -3.0)); vfov = 62.0;
            width = 960; height = 540; spp = 200;
            break;
        case PT_GEN_BATCH_SCENE: {
            // One scene of the 64-scene batch: the random-spheres generator
            // with 10..2000 spheres or the room generator with 2..7
            // subdivisions, a square resolution in {256, 512, 768, 1024} and
            // spp in {4, 16, 64}, all drawn from the scene's seed.
            std::mt19937 rng(static_cast<uint32_t>(params->seed) ^ 0x5bd1e995u);
            auto u = [&rng] { return rng() * 0x1.0p-32; };
            const double pick = u(), size = u(), res = u(), sp = u();
            const int sides[4] = {256, 512, 768, 1024}, spps[3] = {4, 16, 64};
            width = height = sides[std::min(3, int(res * 4))];
            spp = spps[std::min(2, int(sp * 3))];
            aspect = 1.0;
            if (pick < 0.5) {
                random_spheres_scene(b, params->seed, 10 + std::min(1990, int(size * 1991)));
                store(from, p3(13, 2, 3)); store(at, p3(0, 0, 0)); vfov = 20.0;
            } else {
                room_mesh_scene(b, params->seed, 2 + std::min(5, int(size * 6)));
                store(from, p3(0, 0, 3.3)); store(at, p3(0, 0, 0)); vfov = 40.0;
            }
            break;
        }
        default:
            return fail(PT_ERR_INVALID_ARG, "pt_generate: unknown scene kind");
    }
    g->desc.use_bvh = params->use_bvh < 0 ? use_bvh_default : params->use_bvh;
    finish(g.get());
    pt_status st = pt_camera_look_at(from, at, vfov, aspect, &g->cam);
    if (st != PT_OK) return st;
    params->width = width;
    params->height = height;
    params->spp = spp;
    *out = g.release();
    return PT_OK;
}

const pt_scene_desc* pt_generated_desc(const pt_generated* g) { return g ? &g->desc : nullptr; }
const pt_camera* pt_generated_camera(const pt_generated* g) { return g ? &g->cam : nullptr; }
void pt_generated_free(pt_generated* g) { delete g; }

pt_status pt_generate_rays(uint64_t seed, const float lo[3], const float hi[3], size_t n, float* rays) {
    clear_error();
    if (!lo || !hi || (!rays && n)) return fail(PT_ERR_INVALID_ARG, "pt_generate_rays: null pointer");
    std::mt19937_64 rng(seed);
    auto u = [&rng] { return (rng() >> 11) * 0x1.0p-53; };
    for (size_t i = 0; i < n; ++i) {
        const double ox = u(), oy = u(), oz = u(), a = u(), b = u();
        const double z = 1 - 2 * a, phi = 2 * M_PI * b, r = std::sqrt(std::max(0.0, 1 - z * z));
        float* p = rays + 6 * i;
        p[0] = float(lo[0] + (double(hi[0]) - lo[0]) * ox);
        p[1] = float(lo[1] + (double(hi[1]) - lo[1]) * oy);
        p[2] = float(lo[2] + (double(hi[2]) - lo[2]) * oz);
        p[3] = float(r * std::cos(phi));
        p[4] = float(r * std::sin(phi));
        p[5] = float(z);
    }
    return PT_OK;
}

}  // extern "C"
