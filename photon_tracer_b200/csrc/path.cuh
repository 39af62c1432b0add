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

// ---- extended light sampling (PT_FLAG_NEE_EXTENDED; beyond the reference) ---------------
// The density metal scatters into (include/material.hpp:85-91: the mirror
// direction r plus fuzz f times a point uniform in the unit ball, i.e. a point
// uniform in the ball of radius f about r), per unit solid angle at the unit
// direction w: the ball's volume along t*w (t >= 0) weighted by t^2 over the
// ball's volume, (t2^3 - t1^3) / (4 pi f^3) for the chord [t1, t2].
__device__ __forceinline__ float metal_lobe_pdf(V r, float f, V w) {
    const float b = dot(w, r), c = dot(r, r) - f * f;
    const float disc = b * b - c;
    if (!(disc > 0)) return 0;
    const float sq = sqrtf(disc), t2 = b + sq;
    if (!(t2 > 0)) return 0;
    const float t1 = fmaxf(b - sq, 0.0f);
    return (t2 * t2 * t2 - t1 * t1 * t1) / (4 * float(M_PI) * (f * f * f));
}

// Light k of the extended list: first k with u < cdf[k].
__device__ __forceinline__ uint32_t pick_light_ext(const PtSceneDev& S, float u) {
    uint32_t lo = 0, hi = S.n_lights + S.n_tri_lights - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (u < __ldg(S.light_cdf + mid)) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// The extended light sample from the surface rec: a light picked by the
// power-weighted list, a direction toward it (a light sphere's cone as
// direct_light samples it, :41-80; a triangle uniformly over its area), and
// the shadow ray. METAL = false is the matte estimate (albedo / pi times the
// cosine, the albedo applied by the caller); METAL = true the rough-metal one
// (the lobe density at the direction, weighted against the metal's own
// scattered ray by the power heuristic). False when no shadow ray is needed.
template <bool METAL>
__device__ __forceinline__ bool direct_light_ext(const PtSceneDev& S, const Rec& rec, V mirror, float fuzz,
                                                 const Sampler& smp, Rng& rng, Shadow& sh,
                                                 unsigned long long& rays) {
    const uint32_t k = pick_light_ext(S, rng.real());
    V dir, le;
    float cos_surface, pdf_solid, power, t_max;
    bool front = true;
    if (k < S.n_lights) {
        const float4 cr = __ldg(&S.lights[k].cr);
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
        float sp, cp;
        sin_cos(2 * float(M_PI) * s2, sp, cp);
        dir = u * (cp * sin_t) + v * (sp * sin_t) + w * cos_t;
        cos_surface = dot(dir, rec.normal);
        if (cos_surface <= 0) return false;
        float t_light = __int_as_float(0x7f800000);
        if (!sphere_hit(cr, rec.p, dir, 0.001f, t_light)) return false;
        ++rays;
        const V outward = (rec.p + dir * t_light - center) * (1.0f / cr.w);
        front = dot(dir, outward) < 0;
        t_max = t_light * 0.9999f;
        pdf_solid = 1 / (2 * float(M_PI) * one_minus_cos_max);
        le = xyz(__ldg(&S.lights[k].emission));
        power = pt_sphere_light_power(pt_light_luminance(le.x, le.y, le.z), cr.w);
    } else {
        const PtTriLight* L = S.tri_lights + (k - S.n_lights);
        const float4 pa = __ldg(&L->p0_area), e1 = __ldg(&L->e1_er), e2 = __ldg(&L->e2_eg), fe = __ldg(&L->fn_eb);
        float s1, s2;
        smp.sample_2d(1, rng, s1, s2);
        const float sq = sqrtf(s1);
        const V y = xyz(pa) + xyz(e1) * (1 - sq) + xyz(e2) * (s2 * sq);
        const V dv = y - rec.p;
        const float dist2 = dot(dv, dv);
        if (!(dist2 > 0)) return false;
        const float dist = sqrtf(dist2);
        dir = dv * (1.0f / dist);
        const float cos_l = -dot(dir, xyz(fe));
        if (!(cos_l > 0)) return false;  // the emitter's back faces this point: no light
        cos_surface = dot(dir, rec.normal);
        if (cos_surface <= 0) return false;
        ++rays;
        t_max = dist * 0.9999f;
        pdf_solid = dist2 / (pa.w * cos_l);
        le = mk(e1.w, e2.w, fe.w);
        power = pt_triangle_light_power(pt_light_luminance(le.x, le.y, le.z), pa.w);
    }
    const float pdf = (S.pick_uniform + S.pick_power * power) * pdf_solid;
    if (!(pdf > 0) || !(pdf < 3.0e38f)) return false;
    float f;
    if (METAL) {
        const float pb = metal_lobe_pdf(mirror, fuzz, dir);
        const float q = pb / pdf;
        f = q * (1 / (1 + q * q));  // lobe density / light pdf, times the power-heuristic weight
    } else {
        f = cos_surface / float(M_PI) / pdf;
    }
    sh.o = rec.p;
    sh.d = dir;
    sh.t_max = t_max;
    sh.value = front ? le * f : mk(0, 0, 0);
    return front && f > 0;
}

// The extended light-sampling density (pick probability times solid-angle
// density) of the direction d from x that hit the light in rec at distance t.
__device__ __forceinline__ float light_pdf_at_hit(const PtSceneDev& S, const Rec& rec, V x, V d, V le) {
    float pdf_solid, power;
    const float lum = pt_light_luminance(le.x, le.y, le.z);
    if (rec.lkind == 1) {
        const V to_center = xyz(rec.lgeo) - x;
        const float dist2 = dot(to_center, to_center), r2 = rec.lgeo.w * rec.lgeo.w;
        if (dist2 <= r2) return 0;
        const float sin2_max = r2 / dist2;
        const float one_minus_cos_max = sin2_max / (1 + sqrtf(1 - sin2_max));
        pdf_solid = 1 / (2 * float(M_PI) * one_minus_cos_max);
        power = pt_sphere_light_power(lum, rec.lgeo.w);
    } else {
        const float dl = sqrtf(dot(d, d)), dist = rec.t * dl;
        const float cos_l = fabsf(dot(d, xyz(rec.lgeo))) / dl;
        pdf_solid = dist * dist / (rec.lgeo.w * cos_l);
        power = pt_triangle_light_power(lum, rec.lgeo.w);
    }
    return (S.pick_uniform + S.pick_power * power) * pdf_solid;
}

// A path between bounces.
struct Path {
    V o, d;
    V tp, rad;
    int bounce;
    bool sampled;
    float mis_pdf;  // extended light sampling: density of the rough-metal scatter that made d, else 0
};

struct First {
    V albedo, normal;
};

enum : int { STEP_CONTINUE = 0, STEP_DONE = 1 };

// The part of one ray_color iteration after world.hit (:114-146), given the
// record (or a miss). Sets *nee and sh when a shadow ray must be tested, with
// sh.value already multiplied by throughput * attenuation; the caller adds it
// to p.rad if the ray is not blocked. Returns STEP_DONE when the path ends.
template <bool AUX, bool TEX = true, bool EXT = false>
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
    if (rec.front_face && !(p.sampled && rec.sampled_light)) {
        if (EXT && p.mis_pdf > 0 && rec.sampled_light) {
            // a light reached by a rough-metal scatter that also sampled the
            // lights: the power-heuristic weight of the scatter
            const float q = light_pdf_at_hit(S, rec, p.o, p.d, xyz(ef)) / p.mis_pdf;
            p.rad = p.rad + p.tp * (xyz(ef) * (1 / (1 + q * q)));
        } else {
            p.rad = p.rad + p.tp * xyz(ef);
        }
    }
    V att, dir;
    const bool scatters = scatter(mat, type, p.d, rec, smp, rng, att, dir);
    if (TEX && S.has_textures && type == PT_MAT_LAMBERTIAN) {  // albedo * texture->sample(tex_u, tex_v) (:72)
        const uint32_t tex = fbits(mat.ior_flags.z);
        if (tex != PT_NONE) att = att * sample_texture(S, tex, rec.tex_u, rec.tex_v);
    }
    if (AUX && p.bounce == 0)
        first = {scatters && !(flags & PT_MF_TRANSMISSIVE) ? att : mk(1, 1, 1), rec.normal};
    if (EXT) {
        const bool can = S.sample_lights && S.n_lights + S.n_tri_lights > 0 && p.bounce + 1 < depth;
        const float fuzz = mat.emission_fuzz.w;
        p.mis_pdf = 0;
        if (type == PT_MAT_METAL && fuzz > 1e-3f && can) {
            // sampled whether or not the scatter itself is absorbed, so the
            // light estimate does not depend on the scatter's outcome
            const V mirror = reflect(normalize(p.d), rec.normal);
            if (direct_light_ext<true>(S, rec, mirror, fuzz, smp, rng, sh, rays)) {
                nee = true;
                sh.value = (p.tp * att) * sh.value;
            }
            if (scatters) p.mis_pdf = metal_lobe_pdf(mirror, fuzz, normalize(dir));
        }
        if (!scatters) return STEP_DONE;
        p.sampled = (flags & PT_MF_DIFFUSE) && can;
        if (p.sampled && direct_light_ext<false>(S, rec, mk(0, 0, 0), 0.0f, smp, rng, sh, rays)) {
            nee = true;
            sh.value = (p.tp * att) * sh.value;
        }
    } else {
        if (!scatters) return STEP_DONE;
        p.sampled = (flags & PT_MF_DIFFUSE) && S.sample_lights && S.n_lights > 0 && p.bounce + 1 < depth;
        if (p.sampled) {
            if (direct_light_ray(S, rec, smp, rng, sh, rays)) {
                nee = true;
                sh.value = (p.tp * att) * sh.value;
            }
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
template <bool AUX, bool TEX, bool EXT, int N, class Stack>
__device__ __forceinline__ bool query_trip(const PtSceneDev& S, Path& path, int depth, Sampler& smp, Rng& rng,
                                           First& first, float (&pend)[10][N], bool& shadow_pending,
                                           bool& done_after_shadow, Stack& stack, unsigned long long& rays,
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
    if (hit) fill<TEX, EXT>(S, h, path.o, path.d, tq, rec);
    bool nee;
    Shadow sh;
    const bool done = shade<AUX, TEX, EXT>(S, path, hit, rec, depth, smp, rng, first, nee, sh, rays) == STEP_DONE;
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
