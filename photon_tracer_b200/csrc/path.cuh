// The integrator: one bounce of ray_color (include/renderer.hpp:100-149) and
// next event estimation (direct_light, :41-80), split so that the shadow
// ray's occlusion test can run either inline (megakernel) or as its own
// wavefront stage. Nothing here consumes random numbers after the shadow ray
// is made, so resolving it later changes no draw and no float result.
#pragma once
#include "tracer.cuh"

namespace ptd {

struct Cam {
    V origin, llc, horizontal, vertical;
};

// background (include/renderer.hpp:24-29)
__device__ __forceinline__ V background(const PtSceneDev& S, V d) {
    if (!S.sky) return mk(0, 0, 0);
    const V unit = normalize(d);
    const float t = 0.5f * (unit.y + 1);
    return mk(1, 1, 1) * (1 - t) + mk(0.5f, 0.7f, 1.0f) * t;
}

struct Shadow {
    V o, d;
    float t_max;
    V value;  // what direct_light returns when the ray is not blocked
};

// direct_light up to the occlusion test: picks a light, samples its cone and
// builds the shadow ray. Returns false (and the reference returns black)
// when no shadow ray is needed. Counts the shadow ray in *rays the way the
// reference does (:72), i.e. once it reaches the occlusion test.
__device__ __forceinline__ bool direct_light_ray(const PtSceneDev& S, const Rec& rec, const Sampler& smp, Rng& rng,
                                                 Shadow& sh, unsigned long long& rays) {
    const uint32_t n = S.n_lights;
    const uint32_t pick = min(uint32_t(rng.real() * float(n)), n - 1);
    const float4 cr = __ldg(&S.lights[pick].cr);
    const V center = xyz(cr);
    const V to_center = center - rec.p;
    const float dist2 = dot(to_center, to_center), r2 = cr.w * cr.w;
    if (dist2 <= r2) return false;
    const float sin2_max = r2 / dist2;
    const float cos_max = sqrtf(1 - sin2_max);
    const float one_minus_cos_max = sin2_max / (1 + cos_max);
    const V w = div(to_center, sqrtf(dist2));
    const V a = fabsf(w.x) > 0.9f ? mk(0, 1, 0) : mk(1, 0, 0);
    const V u = normalize(cross(w, a)), v = cross(w, u);
    float s1, s2;
    smp.sample_2d(1, rng, s1, s2);
    const float cos_t = 1 - s1 * one_minus_cos_max;
    const float sin_t = sqrtf(fmaxf(0.0f, 1 - cos_t * cos_t));
    const float phi = 2 * float(M_PI) * s2;
    float sp, cp;
    sin_cos(phi, sp, cp);
    const V dir = u * (cp * sin_t) + v * (sp * sin_t) + w * cos_t;
    const float cos_surface = dot(dir, rec.normal);
    if (cos_surface <= 0) return false;
    float t_light = __int_as_float(0x7f800000);
    if (!sphere_hit(cr, rec.p, dir, 0.001f, t_light)) return false;
    ++rays;
    // light.fill + front-face test (:75-77); it does not depend on the
    // occlusion result, so it is decided here.
    const V pl = rec.p + dir * t_light;
    const V outward = (pl - center) * (1.0f / cr.w);
    const bool front = dot(dir, outward) < 0;
    const float pdf = 1 / (2 * float(M_PI) * one_minus_cos_max);
    const float4 em = __ldg(&S.lights[pick].emission);
    sh.o = rec.p;
    sh.d = dir;
    sh.t_max = t_light * 0.9999f;
    sh.value = front ? xyz(em) * (cos_surface / float(M_PI) / pdf * float(n)) : mk(0, 0, 0);
    return front;
}

// A path between bounces.
struct Path {
    V o, d;
    V tp, rad;
    int bounce;
    bool sampled;
};

struct First {
    V albedo, normal;
};

enum : int { STEP_CONTINUE = 0, STEP_DONE = 1 };

// The part of one ray_color iteration after world.hit (:114-146), given the
// record (or a miss). Sets *nee and sh when a shadow ray must be tested, with
// sh.value already multiplied by throughput * attenuation; the caller adds it
// to p.rad if the ray is not blocked. Returns STEP_DONE when the path ends.
template <bool AUX, bool TEX = true>
__device__ __forceinline__ int shade(const PtSceneDev& S, Path& p, bool hit, const Rec& rec, int depth,
                                     const Sampler& smp, Rng& rng, First& first, bool& nee, Shadow& sh,
                                     unsigned long long& rays) {
    nee = false;
    if (!hit) {
        if (AUX && p.bounce == 0) first = {mk(1, 1, 1), mk(0, 0, 0)};
        p.rad = p.rad + p.tp * background(S, p.d);
        return STEP_DONE;
    }
    const PtMaterial* m = S.mat + rec.mat;
    const float4 at = __ldg(&m->albedo_type), ef = __ldg(&m->emission_fuzz), fl = __ldg(&m->ior_flags);
    PtMaterial mat;
    mat.albedo_type = at;
    mat.emission_fuzz = ef;
    mat.ior_flags = fl;
    const uint32_t type = fbits(at.w), flags = fbits(fl.y);
    if (rec.front_face && !(p.sampled && rec.sampled_light)) p.rad = p.rad + p.tp * xyz(ef);
    V att, dir;
    const bool scatters = scatter(mat, type, p.d, rec, smp, rng, att, dir);
    if (TEX && S.has_textures && type == PT_MAT_LAMBERTIAN) {  // albedo * texture->sample(tex_u, tex_v) (:72)
        const uint32_t tex = fbits(mat.ior_flags.z);
        if (tex != PT_NONE) att = att * sample_texture(S, tex, rec.tex_u, rec.tex_v);
    }
    if (AUX && p.bounce == 0)
        first = {scatters && !(flags & PT_MF_TRANSMISSIVE) ? att : mk(1, 1, 1), rec.normal};
    if (!scatters) return STEP_DONE;
    p.sampled = (flags & PT_MF_DIFFUSE) && S.sample_lights && S.n_lights > 0 && p.bounce + 1 < depth;
    if (p.sampled) {
        if (direct_light_ray(S, rec, smp, rng, sh, rays)) {
            nee = true;
            sh.value = (p.tp * att) * sh.value;
        }
    }
    p.tp = p.tp * att;
    p.o = rec.p;
    p.d = dir;
    // Russian roulette (:140-146)
    if (p.bounce + 1 >= 3) {
        const float q = fmaxf(p.tp.x, fmaxf(p.tp.y, p.tp.z));
        if (q < 1) {
            if (rng.real() >= q) return STEP_DONE;
            p.tp = div(p.tp, q);
        }
    }
    p.bounce++;
    return p.bounce >= depth ? STEP_DONE : STEP_CONTINUE;
}

// One loop trip of a persistent kernel that traces ONE query per trip for a
// scene without instances: the path's next closest hit (then its shading),
// or the shadow ray the previous trip's shading made, which is resolved
// before the path continues. Nothing between making the shadow ray and
// resolving it consumes random numbers or touches the path's sums, so the
// results are those of the inline form. The pending shadow ray (origin,
// direction, t_max, unblocked value) of each thread sits in shared memory,
// column threadIdx.x of pend. Returns true when the path has ended.
template <bool AUX, bool TEX, int N>
__device__ __forceinline__ bool query_trip(const PtSceneDev& S, Path& path, int depth, Sampler& smp, Rng& rng,
                                           First& first, float (&pend)[10][N], bool& shadow_pending,
                                           bool& done_after_shadow, StackEntry* stack, unsigned long long& rays,
                                           bool& overflow) {
    const int t = threadIdx.x;
    const bool any = shadow_pending;
    V qo, qd;
    float tq;
    if (any) {
        qo = mk(pend[0][t], pend[1][t], pend[2][t]);
        qd = mk(pend[3][t], pend[4][t], pend[5][t]);
        tq = pend[6][t];
    } else {
        ++rays;
        smp.set_bounce(path.bounce);
        qo = path.o;
        qd = path.d;
        tq = 1000.0f;
    }
    Hit h;
    if (!query_flat(S, qo, qd, 0.001f, tq, any, h, stack)) {
        overflow = true;
        h.kind = PT_HIT_NONE;
    }
    if (any) {
        if (h.kind == PT_HIT_NONE) path.rad = path.rad + mk(pend[7][t], pend[8][t], pend[9][t]);
        shadow_pending = false;
        return done_after_shadow;
    }
    const bool hit = h.kind != PT_HIT_NONE;
    Rec rec;
    if (hit) fill<TEX>(S, h, path.o, path.d, tq, rec);
    bool nee;
    Shadow sh;
    const bool done = shade<AUX, TEX>(S, path, hit, rec, depth, smp, rng, first, nee, sh, rays) == STEP_DONE;
    if (!nee) return done;
    pend[0][t] = sh.o.x;
    pend[1][t] = sh.o.y;
    pend[2][t] = sh.o.z;
    pend[3][t] = sh.d.x;
    pend[4][t] = sh.d.y;
    pend[5][t] = sh.d.z;
    pend[6][t] = sh.t_max;
    pend[7][t] = sh.value.x;
    pend[8][t] = sh.value.y;
    pend[9][t] = sh.value.z;
    shadow_pending = true;
    done_after_shadow = done;
    return false;
}

// luminance (include/renderer.hpp:364)
__device__ __forceinline__ float luminance(V c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

}  // namespace ptd
