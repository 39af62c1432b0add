/*
 * pt_oracle.c -- TEST INFRASTRUCTURE, not part of the product.
 *
 * A plain-C, single-threaded CPU restatement of photon_tracer's render hot
 * path, used only to check results in tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py. Nothing in the product links or calls it.
 *
 * Each function names the reference function it restates (photon_tracer,
 * include/<file>:<lines>). It is compiled with -ffp-contract=off, like the
 * reference (built without FMA), so on the same machine it reproduces the
 * reference's floats exactly; the tests pin it against the reference itself
 * (oracle/_ref, built from the reference's own headers) and against the
 * reference's statistical fixtures.
 *
 * Inputs are the scene description of include/photon_cuda.h plus the BVHs
 * (bvh::node layout) for the flat tree, the instance tree and each mesh.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/photon_cuda.h"

#define PO_STACK (3 * 64 + 1) /* bvh.hpp:66-68 */

typedef struct {
    float x, y, z;
} v3;

static v3 mk(float x, float y, float z) {
    v3 r = {x, y, z};
    return r;
}
static v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
static v3 mul(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static v3 scl(v3 a, float t) { return mk(a.x * t, a.y * t, a.z * t); }
static float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }                 /* vec3.hpp:91-93 */
static v3 cross(v3 a, v3 b) {                                                              /* vec3.hpp:114-118 */
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static v3 normalize(v3 a) { /* vec3.hpp:95-98 */
    float len = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
    return mk(a.x / len, a.y / len, a.z / len);
}
static v3 vdiv(v3 a, float t) { return scl(a, 1 / t); } /* vec3.hpp:87-89 */
static v3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }

/* ---- scene ---------------------------------------------------------------------- */
typedef struct {
    const pt_bvh_node* nodes;
    uint32_t n_nodes;
    const uint32_t* order;
} tree;

typedef struct po_scene {
    pt_scene_desc d;
    tree flat, inst;
    tree* mesh;
    uint32_t* lights;
    uint32_t n_lights;
    float** texels; /* per texture: linear RGB (image_texture's texels, texture.hpp:13-21) */
    /* The extended light list (PT_FLAG_NEE_EXTENDED, beyond the reference):
     * emissive flat triangles of positive area, after the light spheres, and
     * the cumulative pick probabilities of all of them. */
    uint32_t* tri_lights;
    float* tri_area;
    uint32_t n_tri_lights;
    float* light_cdf;
    float pick_uniform, pick_power;
} po_scene;

static int emits(const pt_material* m) { return m->emission[0] > 0 || m->emission[1] > 0 || m->emission[2] > 0; }

/* Power of a light for the extended pick: luminance of the emission times
 * the area (4 pi r^2 for a sphere), 0 when not positive and finite; half the
 * pick probability is uniform over the lights, half in proportion to power. */
static float light_lum(const float* e) { return 0.2126f * e[0] + 0.7152f * e[1] + 0.0722f * e[2]; }
static float sphere_power(float lum, float r) {
    const float p = lum * (4.0f * 3.14159265f * (r * r));
    return p > 0.0f && p < 3.0e38f ? p : 0.0f;
}
static float tri_area(const float* a, const float* b) {
    const float cx = a[1] * b[2] - a[2] * b[1], cy = a[2] * b[0] - a[0] * b[2], cz = a[0] * b[1] - a[1] * b[0];
    return 0.5f * sqrtf(cx * cx + cy * cy + cz * cz);
}
static float tri_power(float lum, float area) {
    const float p = lum * area;
    return p > 0.0f && p < 3.0e38f ? p : 0.0f;
}

po_scene* po_scene_create(const pt_scene_desc* d, const pt_bvh* flat, const pt_bvh* inst, const pt_bvh* meshes) {
    po_scene* s = (po_scene*)calloc(1, sizeof(po_scene));
    uint32_t i;
    s->d = *d;
    if (flat) {
        s->flat.nodes = flat->nodes;
        s->flat.n_nodes = flat->n_nodes;
        s->flat.order = flat->order;
    }
    if (inst) {
        s->inst.nodes = inst->nodes;
        s->inst.n_nodes = inst->n_nodes;
        s->inst.order = inst->order;
    }
    s->mesh = (tree*)calloc(d->n_meshes ? d->n_meshes : 1, sizeof(tree));
    for (i = 0; i < d->n_meshes; ++i) {
        s->mesh[i].nodes = meshes[i].nodes;
        s->mesh[i].n_nodes = meshes[i].n_nodes;
        s->mesh[i].order = meshes[i].order;
    }
    /* image_texture (texture.hpp:13-21): sRGB bytes to linear through a 256-entry table */
    s->texels = (float**)calloc(d->n_textures ? d->n_textures : 1, sizeof(float*));
    if (d->n_textures) {
        float table[256];
        int v;
        for (v = 0; v < 256; ++v) {
            const float c = v / 255.0f;
            table[v] = c <= 0.04045f ? c / 12.92f : powf((c + 0.055f) / 1.055f, 2.4f);
        }
        for (i = 0; i < d->n_textures; ++i) {
            const size_t n = 3 * (size_t)d->textures[i].width * (size_t)d->textures[i].height;
            size_t k;
            s->texels[i] = (float*)malloc((n ? n : 1) * sizeof(float));
            for (k = 0; k < n; ++k) s->texels[i][k] = table[d->textures[i].rgb[k]];
        }
    }
    /* geometry::build's light list (geometry.hpp:75-77) */
    s->lights = (uint32_t*)calloc(d->n_spheres ? d->n_spheres : 1, sizeof(uint32_t));
    if (d->lights) {
        memcpy(s->lights, d->lights, d->n_lights * sizeof(uint32_t));
        s->n_lights = d->n_lights;
    } else {
        for (i = 0; i < d->n_spheres; ++i)
            if (emits(&d->materials[d->spheres[i].material])) s->lights[s->n_lights++] = i;
    }
    /* the extended list: the light spheres, then every emissive flat triangle of positive area */
    {
        uint32_t n, k;
        float* power;
        double total = 0, sum = 0, acc = 0;
        s->tri_lights = (uint32_t*)calloc(d->n_triangles ? d->n_triangles : 1, sizeof(uint32_t));
        s->tri_area = (float*)calloc(d->n_triangles ? d->n_triangles : 1, sizeof(float));
        for (i = 0; i < d->n_triangles; ++i) {
            const pt_triangle* t = &d->triangles[i];
            float a;
            if (!emits(&d->materials[t->material])) continue;
            a = tri_area(t->e1, t->e2);
            if (!(a > 0.0f) || !(a < 3.0e38f)) continue;
            s->tri_area[s->n_tri_lights] = a;
            s->tri_lights[s->n_tri_lights++] = i;
        }
        n = s->n_lights + s->n_tri_lights;
        power = (float*)calloc(n ? n : 1, sizeof(float));
        for (k = 0; k < s->n_lights; ++k) {
            const pt_sphere* L = &d->spheres[s->lights[k]];
            power[k] = sphere_power(light_lum(d->materials[L->material].emission), L->radius);
        }
        for (k = 0; k < s->n_tri_lights; ++k)
            power[s->n_lights + k] = tri_power(light_lum(d->materials[d->triangles[s->tri_lights[k]].material].emission),
                                               s->tri_area[k]);
        s->light_cdf = (float*)calloc(n ? n : 1, sizeof(float));
        if (n) {
            for (k = 0; k < n; ++k) total += power[k];
            if (total > 0) {
                s->pick_uniform = (float)(0.5 / (double)n);
                s->pick_power = (float)(0.5 / total);
            } else {
                s->pick_uniform = (float)(1.0 / (double)n);
                s->pick_power = 0;
            }
            for (k = 0; k < n; ++k) sum += (double)(s->pick_uniform + s->pick_power * power[k]);
            for (k = 0; k < n; ++k) {
                acc += (double)(s->pick_uniform + s->pick_power * power[k]);
                s->light_cdf[k] = k + 1 == n ? 1.0f : (float)(acc / sum);
            }
        }
        free(power);
    }
    return s;
}

void po_scene_destroy(po_scene* s) {
    uint32_t i;
    if (!s) return;
    for (i = 0; i < s->d.n_textures; ++i) free(s->texels[i]);
    free(s->texels);
    free(s->mesh);
    free(s->lights);
    free(s->tri_lights);
    free(s->tri_area);
    free(s->light_cdf);
    free(s);
}

/* ---- primitives ------------------------------------------------------------------ */
/* sphere::intersect<float> (sphere.hpp:25-48) */
static int sphere_hit(const pt_sphere* s, v3 o, v3 d, float t_min, float* t_max) {
    float ox = o.x - s->center[0], oy = o.y - s->center[1], oz = o.z - s->center[2];
    float a = d.x * d.x + d.y * d.y + d.z * d.z;
    float half_b = ox * d.x + oy * d.y + oz * d.z;
    float c = ox * ox + oy * oy + oz * oz - s->radius * s->radius;
    float disc = half_b * half_b - a * c, sq, root;
    if (disc < 0) return 0;
    sq = sqrtf(disc);
    root = (-half_b - sq) / a;
    if (root < t_min || root > *t_max) {
        root = (-half_b + sq) / a;
        if (root < t_min || root > *t_max) return 0;
    }
    *t_max = root;
    return 1;
}

/* sphere::intersect<double> (sphere.hpp:25-48 with P = double) */
static int sphere_hit_double(const pt_sphere* s, v3 o, v3 d, float t_min, float* t_max) {
    double ox = (double)o.x - s->center[0], oy = (double)o.y - s->center[1], oz = (double)o.z - s->center[2];
    double dx = d.x, dy = d.y, dz = d.z;
    double a = dx * dx + dy * dy + dz * dz;
    double half_b = ox * dx + oy * dy + oz * dz;
    double c = ox * ox + oy * oy + oz * oz - (double)s->radius * s->radius;
    double disc = half_b * half_b - a * c, sq, root;
    if (disc < 0) return 0;
    sq = sqrt(disc);
    root = (-half_b - sq) / a;
    if (root < t_min || root > *t_max) {
        root = (-half_b + sq) / a;
        if (root < t_min || root > *t_max) return 0;
    }
    *t_max = (float)root;
    return 1;
}

/* triangle::intersect (triangle.hpp:40-61) */
static int tri_hit(const pt_triangle* tr, v3 o, v3 d, float t_min, float* t_max, float* uo, float* vo) {
    v3 e1 = ld3(tr->e1), e2 = ld3(tr->e2);
    v3 pvec = cross(d, e2), tvec, qvec;
    float det = dot(e1, pvec), inv_det, u, v, t;
    if (fabsf(det) < 1e-12f) return 0;
    inv_det = 1 / det;
    tvec = sub(o, ld3(tr->p0));
    u = dot(tvec, pvec) * inv_det;
    if (u < 0 || u > 1) return 0;
    qvec = cross(tvec, e1);
    v = dot(d, qvec) * inv_det;
    if (v < 0 || u + v > 1) return 0;
    t = dot(e2, qvec) * inv_det;
    if (t < t_min || t > *t_max) return 0;
    *t_max = t;
    *uo = u;
    *vo = v;
    return 1;
}

/* affine::vector / point / transposed (transform.hpp:15-27) */
static v3 aff_vector(const pt_affine* x, v3 v) {
    return mk(x->m[0][0] * v.x + x->m[0][1] * v.y + x->m[0][2] * v.z,
              x->m[1][0] * v.x + x->m[1][1] * v.y + x->m[1][2] * v.z,
              x->m[2][0] * v.x + x->m[2][1] * v.y + x->m[2][2] * v.z);
}
static v3 aff_point(const pt_affine* x, v3 p) { return add(aff_vector(x, p), ld3(x->t)); }
static v3 aff_transposed(const pt_affine* x, v3 v) {
    return mk(x->m[0][0] * v.x + x->m[1][0] * v.y + x->m[2][0] * v.z,
              x->m[0][1] * v.x + x->m[1][1] * v.y + x->m[2][1] * v.z,
              x->m[0][2] * v.x + x->m[1][2] * v.y + x->m[2][2] * v.z);
}

/* ---- traversal (bvh.hpp:57-106) --------------------------------------------------- */
typedef struct {
    uint64_t nodes, order, tris, spheres, insts;
} counts;

typedef struct {
    uint32_t first, count;
    float t;
} entry;

/* leaf callback: tests primitives order[first..first+count) */
typedef void (*leaf_fn)(void* ctx, uint32_t prim, float* t_max);

static float sse_min(float a, float b) { return a < b ? a : b; } /* simd4.hpp:15 (_mm_min_ps) */
static float sse_max(float a, float b) { return a > b ? a : b; } /* simd4.hpp:16 (_mm_max_ps) */

static void traverse(const tree* tr, v3 o, v3 d, float t_min, float* t_max, counts* cnt, leaf_fn test, void* ctx) {
    entry stack[PO_STACK];
    int top = 0;
    float ix, iy, iz;
    if (!tr->nodes || tr->n_nodes == 0) return;
    ix = 1 / d.x;
    iy = 1 / d.y;
    iz = 1 / d.z;
    stack[top].first = 0;
    stack[top].count = 0;
    stack[top].t = t_min;
    ++top;
    while (top > 0) {
        entry e = stack[--top], hit[4];
        const pt_bvh_node* nd;
        float tn[4];
        int mask = 0, c, n = 0, k;
        uint32_t i;
        if (e.t >= *t_max) continue;
        if (e.count > 0) {
            for (i = e.first; i < e.first + e.count; ++i) {
                if (cnt) cnt->order++;
                test(ctx, tr->order[i], t_max);
            }
            continue;
        }
        nd = &tr->nodes[e.first];
        if (cnt) cnt->nodes++;
        for (c = 0; c < 4; ++c) {
            float x0 = (nd->lo[0][c] - o.x) * ix, x1 = (nd->hi[0][c] - o.x) * ix;
            float y0 = (nd->lo[1][c] - o.y) * iy, y1 = (nd->hi[1][c] - o.y) * iy;
            float z0 = (nd->lo[2][c] - o.z) * iz, z1 = (nd->hi[2][c] - o.z) * iz;
            float tnear = sse_max(sse_max(sse_min(x0, x1), sse_min(y0, y1)), sse_max(sse_min(z0, z1), t_min));
            float tfar = sse_min(sse_min(sse_max(x0, x1), sse_max(y0, y1)), sse_min(sse_max(z0, z1), *t_max));
            tn[c] = tnear;
            if (tnear <= tfar) mask |= 1 << c;
        }
        if (mask == 0) continue;
        /* insertion sort, farthest first (bvh.hpp:93-104) */
        for (c = 0; c < 4; ++c) {
            entry h;
            if (!(mask & (1 << c))) continue;
            h.first = nd->first[c];
            h.count = nd->count[c];
            h.t = tn[c];
            k = n++;
            for (; k > 0 && hit[k - 1].t < h.t; --k) hit[k] = hit[k - 1];
            hit[k] = h;
        }
        /* bvh.hpp pushes without a bound; 3 * depth + 1 entries suffice for
           every ray whose slab values are not NaN. A NaN origin or direction
           makes every child test pass, empty children (first 0, count 0)
           included, which re-enter the root without end: the reference then
           overruns its stack and crashes. Here the walk stops instead. */
        if (top + n > PO_STACK) return;
        for (k = 0; k < n; ++k) stack[top++] = hit[k];
    }
}

/* ---- geometry::hit (geometry.hpp:111-152) -------------------------------------- */
typedef struct {
    const po_scene* s;
    v3 o, d;
    float t_min;
    uint32_t kind, index, sub;
    float u, v;
    counts* cnt;
    /* instance walk (hit_instance, :212-229) */
    const pt_triangle* mtris;
    v3 lo, ld;
    int found, any_hit, blocked;
    uint32_t tri;
    float hu, hv;
} hctx;

static void test_flat(void* p, uint32_t prim, float* t_far) {
    hctx* c = (hctx*)p;
    const pt_scene_desc* d = &c->s->d;
    if (prim < d->n_spheres) {
        if (c->cnt) c->cnt->spheres++;
        if (sphere_hit(&d->spheres[prim], c->o, c->d, c->t_min, t_far)) {
            c->kind = PT_HIT_SPHERE;
            c->index = prim;
        }
    } else {
        if (c->cnt) c->cnt->tris++;
        if (tri_hit(&d->triangles[prim - d->n_spheres], c->o, c->d, c->t_min, t_far, &c->u, &c->v)) {
            c->kind = PT_HIT_TRIANGLE;
            c->index = prim - d->n_spheres;
        }
    }
}

static void test_mesh_tri(void* p, uint32_t tri, float* t_mesh) {
    hctx* c = (hctx*)p;
    if (c->found && c->any_hit) return;
    if (c->cnt) c->cnt->tris++;
    if (tri_hit(&c->mtris[tri], c->lo, c->ld, c->t_min, t_mesh, &c->hu, &c->hv)) {
        c->found = 1;
        c->tri = tri;
        if (c->any_hit) *t_mesh = c->t_min;
    }
}

/* hit_instance (geometry.hpp:212-229): returns found, writes t. */
static int hit_instance(hctx* c, uint32_t k, float t_far, float* t_out) {
    const pt_instance* in = &c->s->d.instances[k];
    const pt_mesh* m = &c->s->d.meshes[in->mesh];
    float ht = t_far;
    if (c->cnt) c->cnt->insts++;
    c->mtris = m->triangles;
    c->lo = aff_point(&in->to_object, c->o);
    c->ld = aff_vector(&in->to_object, c->d);
    c->found = 0;
    c->hu = 0;
    c->hv = 0;
    traverse(&c->s->mesh[in->mesh], c->lo, c->ld, c->t_min, &ht, c->cnt, test_mesh_tri, c);
    *t_out = ht;
    return c->found;
}

static void test_instance(void* p, uint32_t k, float* t_far) {
    hctx* c = (hctx*)p;
    float t;
    c->any_hit = 0;
    if (hit_instance(c, k, *t_far, &t)) {
        c->kind = PT_HIT_INSTANCE;
        c->index = k;
        *t_far = t;
        c->u = c->hu;
        c->v = c->hv;
        c->sub = c->tri;
    }
}

/* Closest hit: kind/index/sub/u/v as geometry::hit decides them; t_max updated. */
static void closest(const po_scene* s, v3 o, v3 d, float t_min, float* t_max, hctx* c, counts* cnt) {
    const pt_scene_desc* D = &s->d;
    uint32_t i;
    memset(c, 0, sizeof(*c));
    c->s = s;
    c->o = o;
    c->d = d;
    c->t_min = t_min;
    c->cnt = cnt;
    c->kind = PT_HIT_NONE;
    for (i = 0; i < D->n_large_spheres; ++i)
        if (sphere_hit_double(&D->large_spheres[i], o, d, t_min, t_max)) {
            c->kind = PT_HIT_LARGE;
            c->index = i;
        }
    if (D->use_bvh) {
        traverse(&s->flat, o, d, t_min, t_max, cnt, test_flat, c);
        if (D->n_instances) traverse(&s->inst, o, d, t_min, t_max, cnt, test_instance, c);
    } else {
        uint32_t n = D->n_spheres + D->n_triangles, p, k;
        for (p = 0; p < n; ++p) {
            if (cnt) cnt->order++;
            test_flat(c, p, t_max);
        }
        for (k = 0; k < D->n_instances; ++k) {
            if (cnt) cnt->order++;
            test_instance(c, k, t_max);
        }
    }
}

/* geometry::occluded (geometry.hpp:156-190) */
static void occ_flat(void* p, uint32_t prim, float* t_far) {
    hctx* c = (hctx*)p;
    const pt_scene_desc* d = &c->s->d;
    float t = *t_far, u, v;
    if (c->blocked) return;
    if (prim < d->n_spheres) {
        if (c->cnt) c->cnt->spheres++;
        c->blocked = sphere_hit(&d->spheres[prim], c->o, c->d, c->t_min, &t);
    } else {
        if (c->cnt) c->cnt->tris++;
        c->blocked = tri_hit(&d->triangles[prim - d->n_spheres], c->o, c->d, c->t_min, &t, &u, &v);
    }
    if (c->blocked) *t_far = c->t_min;
}

static void occ_instance(void* p, uint32_t k, float* t_far) {
    hctx* c = (hctx*)p;
    float t;
    if (c->blocked) return;
    c->any_hit = 1;
    c->blocked = hit_instance(c, k, *t_far, &t);
    if (c->blocked) *t_far = c->t_min;
}

static int occluded(const po_scene* s, v3 o, v3 d, float t_min, float t_max, counts* cnt) {
    const pt_scene_desc* D = &s->d;
    hctx c;
    float t_far;
    uint32_t i;
    for (i = 0; i < D->n_large_spheres; ++i) {
        float t = t_max;
        if (sphere_hit_double(&D->large_spheres[i], o, d, t_min, &t)) return 1;
    }
    memset(&c, 0, sizeof(c));
    c.s = s;
    c.o = o;
    c.d = d;
    c.t_min = t_min;
    c.cnt = cnt;
    t_far = t_max;
    if (D->use_bvh) {
        traverse(&s->flat, o, d, t_min, &t_far, cnt, occ_flat, &c);
        if (!c.blocked && D->n_instances) {
            t_far = t_max;
            traverse(&s->inst, o, d, t_min, &t_far, cnt, occ_instance, &c);
        }
    } else {
        uint32_t n = D->n_spheres + D->n_triangles, p, k;
        for (p = 0; p < n && !c.blocked; ++p) occ_flat(&c, p, &t_far);
        for (k = 0; k < D->n_instances && !c.blocked; ++k) occ_instance(&c, k, &t_far);
    }
    return c.blocked;
}

/* ---- hit records (hittable.hpp, sphere.hpp:50-58, triangle.hpp:63-74, geometry.hpp:141-151, 234-244) */
typedef struct {
    v3 p, normal;
    float t;
    int front_face, sampled_light;
    uint32_t mat;
    float tex_u, tex_v;
    /* extended light sampling: 1 a light sphere (lgeo = center, lw = radius),
     * 2 an emissive flat triangle (lgeo = face normal, lw = area), else 0 */
    int lkind;
    v3 lgeo;
    float lw;
} rec_t;

static void fill_sphere(const pt_sphere* s, v3 o, v3 d, float t, rec_t* r) {
    v3 outward;
    r->t = t;
    r->p = add(o, scl(d, t));
    outward = scl(sub(r->p, ld3(s->center)), 1 / s->radius);
    r->front_face = dot(d, outward) < 0;
    r->normal = r->front_face ? outward : neg(outward);
    r->mat = s->material;
}

static void fill_triangle(const pt_triangle* tr, v3 o, v3 d, float t, float u, float v, rec_t* r) {
    v3 n;
    r->t = t;
    r->p = add(o, scl(d, t));
    r->front_face = dot(d, ld3(tr->face_normal)) < 0;
    n = normalize(add(add(scl(ld3(tr->n0), 1 - u - v), scl(ld3(tr->n1), u)), scl(ld3(tr->n2), v)));
    r->normal = r->front_face ? n : neg(n);
    r->mat = tr->material;
    r->tex_u = tr->uv[0] * (1 - u - v) + tr->uv[2] * u + tr->uv[4] * v;
    r->tex_v = tr->uv[1] * (1 - u - v) + tr->uv[3] * u + tr->uv[5] * v;
}

/* image_texture::sample (texture.hpp:25-33) */
static v3 texel(const po_scene* s, uint32_t k, int x, int y) {
    const int w = s->d.textures[k].width, h = s->d.textures[k].height;
    const float* t;
    x = ((x % w) + w) % w;
    y = ((y % h) + h) % h;
    t = &s->texels[k][3 * ((size_t)y * w + x)];
    return mk(t[0], t[1], t[2]);
}
static v3 sample_texture(const po_scene* s, uint32_t k, float u, float v) {
    const float x = (u - floorf(u)) * (float)s->d.textures[k].width - 0.5f;
    const float y = (1 - (v - floorf(v))) * (float)s->d.textures[k].height - 0.5f;
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const float fx = x - (float)x0, fy = y - (float)y0;
    return add(add(add(scl(texel(s, k, x0, y0), (1 - fx) * (1 - fy)), scl(texel(s, k, x0 + 1, y0), fx * (1 - fy))),
                   scl(texel(s, k, x0, y0 + 1), (1 - fx) * fy)),
               scl(texel(s, k, x0 + 1, y0 + 1), fx * fy));
}

static int hit(const po_scene* s, v3 o, v3 d, float t_min, float t_max, rec_t* r, counts* cnt, int ext) {
    const pt_scene_desc* D = &s->d;
    hctx c;
    closest(s, o, d, t_min, &t_max, &c, cnt);
    r->sampled_light = 0;
    r->lkind = 0;
    r->tex_u = 0;
    r->tex_v = 0;
    switch (c.kind) {
        case PT_HIT_LARGE: fill_sphere(&D->large_spheres[c.index], o, d, t_max, r); return 1;
        case PT_HIT_SPHERE:
            fill_sphere(&D->spheres[c.index], o, d, t_max, r);
            r->sampled_light = D->sample_lights && emits(&D->materials[r->mat]);
            if (ext && r->sampled_light) {
                r->lkind = 1;
                r->lgeo = ld3(D->spheres[c.index].center);
                r->lw = D->spheres[c.index].radius;
            }
            return 1;
        case PT_HIT_TRIANGLE: {
            const pt_triangle* tr = &D->triangles[c.index];
            fill_triangle(tr, o, d, t_max, c.u, c.v, r);
            if (ext && D->sample_lights && emits(&D->materials[r->mat])) {
                const float a = tri_area(tr->e1, tr->e2);
                if (a > 0.0f && a < 3.0e38f) {
                    r->sampled_light = 1;
                    r->lkind = 2;
                    r->lgeo = ld3(tr->face_normal);
                    r->lw = a;
                }
            }
            return 1;
        }
        case PT_HIT_INSTANCE: {
            const pt_instance* in = &D->instances[c.index];
            v3 lo = aff_point(&in->to_object, o), ldir = aff_vector(&in->to_object, d);
            fill_triangle(&D->meshes[in->mesh].triangles[c.sub], lo, ldir, t_max, c.u, c.v, r);
            r->p = add(o, scl(d, t_max));
            r->normal = normalize(aff_transposed(&in->to_object, r->normal));
            if (in->material != PT_NO_MATERIAL) r->mat = in->material;
            return 1;
        }
        default: return 0;
    }
}

/* ---- random numbers (vec3.hpp:11-52) and the sampler (sampler.hpp) ------------- */
typedef struct {
    uint64_t s[4];
} rng_t;

static void rng_seed(rng_t* r, uint64_t seed) {
    int k;
    for (k = 0; k < 4; ++k) {
        uint64_t z = (seed += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        r->s[k] = z ^ (z >> 31);
    }
}
static uint64_t rng_next(rng_t* r) {
    uint64_t* s = r->s;
    uint64_t result = s[0] + s[3], t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = (s[3] << 45) | (s[3] >> 19);
    return result;
}
static float rng_real(rng_t* r) { return (float)(rng_next(r) >> 40) * 0x1.0p-24f; }

/* The per-(pixel, sample) stream of PT_RNG_SAMPLE (the library's production mode). */
uint64_t po_sample_stream_seed(uint64_t seed, int i, int j, uint32_t s) {
    uint64_t x = seed ^ (((uint64_t)(uint32_t)j << 32) | (uint32_t)i);
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x ^ ((uint64_t)s * 0xd6e8feb86659fd93ull);
}

static uint32_t reverse_bits(uint32_t x) {
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
    x = ((x >> 8) & 0x00ff00ffu) | ((x & 0x00ff00ffu) << 8);
    return (x >> 16) | (x << 16);
}
static uint32_t hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
static uint32_t lk_permute(uint32_t x, uint32_t seed) {
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
/* sobol_1_tables (sampler.hpp:67-94), built once */
static uint32_t sobol_tab[4][256];
static int sobol_ready = 0;
static void sobol_init(void) {
    uint32_t v[32];
    int k, byte;
    uint32_t b;
    if (sobol_ready) return;
    v[0] = 1u << 31;
    for (k = 1; k < 32; ++k) v[k] = v[k - 1] ^ (v[k - 1] >> 1);
    for (byte = 0; byte < 4; ++byte)
        for (b = 0; b < 256; ++b) {
            uint32_t r = 0;
            for (k = 0; k < 8; ++k)
                if (b & (1u << k)) r ^= v[8 * byte + k];
            sobol_tab[byte][b] = reverse_bits(r);
        }
    sobol_ready = 1;
}
static uint32_t sobol_1_reversed(uint32_t i) {
    return sobol_tab[0][i & 255] ^ sobol_tab[1][(i >> 8) & 255] ^ sobol_tab[2][(i >> 16) & 255] ^ sobol_tab[3][i >> 24];
}

typedef struct {
    uint32_t pixel_seed, index;
    int base;
} sampler_t;

static void begin_sample(sampler_t* q, uint64_t seed, int i, int j, uint32_t index) { /* sampler.hpp:98-104 */
    q->pixel_seed = hash_u32((uint32_t)i * 0x9e3779b1u ^
                             hash_u32((uint32_t)j ^ hash_u32((uint32_t)seed ^ (uint32_t)(seed >> 32))));
    q->index = index;
    q->base = 0;
}
static void sample_2d(const sampler_t* q, rng_t* r, int pair_offset, float* a, float* b) { /* sampler.hpp:107-124 */
    int pair = q->base + pair_offset;
    uint32_t seed, i, x, y;
    if (pair > 4) {
        *a = rng_real(r);
        *b = rng_real(r);
        return;
    }
    seed = hash_u32(q->pixel_seed + (uint32_t)pair * 0x68bc21ebu);
    i = reverse_bits(lk_permute(reverse_bits(q->index), seed));
    x = reverse_bits(lk_permute(i, seed ^ 0xa511e9b3u));
    y = reverse_bits(lk_permute(sobol_1_reversed(i), seed ^ 0x63d83595u));
    *a = (float)(x >> 8) * 0x1.0p-24f;
    *b = (float)(y >> 8) * 0x1.0p-24f;
}

/* Exposed for the sampler known-answer tests: (a, b) for one pair. */
void po_sample_2d(uint64_t seed, int i, int j, uint32_t index, int bounce, int pair_offset, float out[2]) {
    sampler_t q;
    rng_t r;
    sobol_init();
    begin_sample(&q, seed, i, j, index);
    if (bounce >= 0) q.base = 1 + 2 * bounce;
    rng_seed(&r, 1);
    sample_2d(&q, &r, pair_offset, &out[0], &out[1]);
}

/* ---- materials (material.hpp) ------------------------------------------------------- */
static v3 reflect(v3 v, v3 n) { return sub(v, scl(n, 2 * dot(v, n))); }
static v3 refract(v3 uv, v3 n, float ratio) {
    float cos_theta = fminf(dot(neg(uv), n), 1.0f);
    v3 r_perp = scl(add(uv, scl(n, cos_theta)), ratio);
    v3 r_par = scl(n, -sqrtf(fabsf(1 - dot(r_perp, r_perp))));
    return add(r_perp, r_par);
}
/* random_in_unit_sphere (vec3.hpp:121-127); GCC evaluates vec3::random's three
 * constructor arguments right to left, so z is drawn first. */
static v3 random_in_unit_sphere(rng_t* r) {
    for (;;) {
        float z = -1 + 2 * rng_real(r);
        float y = -1 + 2 * rng_real(r);
        float x = -1 + 2 * rng_real(r);
        v3 p = mk(x, y, z);
        if (dot(p, p) >= 1) continue;
        return p;
    }
}

static int scatter(const pt_material* m, v3 d_in, const rec_t* rec, const sampler_t* q, rng_t* r, v3* att, v3* dir) {
    if (m->type == PT_MAT_LAMBERTIAN) { /* :59-74 */
        float a, b, rr, phi, sign, p, qq;
        v3 n = rec->normal, t1, t2;
        sample_2d(q, r, 0, &a, &b);
        rr = sqrtf(a);
        phi = 2 * (float)M_PI * b;
        sign = copysignf(1.0f, n.z);
        p = -1 / (sign + n.z);
        qq = n.x * n.y * p;
        t1 = mk(1 + sign * n.x * n.x * p, sign * qq, -sign * n.x);
        t2 = mk(qq, sign + n.y * n.y * p, -n.y);
        *dir = add(add(scl(t1, rr * cosf(phi)), scl(t2, rr * sinf(phi))), scl(n, sqrtf(fmaxf(0.0f, 1 - a))));
        *att = ld3(m->albedo);
        return 1;
    }
    if (m->type == PT_MAT_METAL) { /* :85-91; the constructor keeps fuzz = f < 1 ? f : 1 (:83) */
        const float fuzz = m->fuzz < 1 ? m->fuzz : 1;
        v3 refl = reflect(normalize(d_in), rec->normal);
        *dir = add(refl, scl(random_in_unit_sphere(r), fuzz));
        *att = ld3(m->albedo);
        return dot(*dir, rec->normal) > 0;
    }
    if (m->type == PT_MAT_DIELECTRIC) { /* :113-136 */
        float ratio = rec->front_face ? (1 / m->ior) : m->ior;
        v3 unit = normalize(d_in);
        float cos_theta = fminf(dot(neg(unit), rec->normal), 1.0f);
        float sin_theta = sqrtf(1 - cos_theta * cos_theta);
        int refl = ratio * sin_theta > 1;
        *att = mk(1, 1, 1);
        if (!refl) {
            float r0 = (1 - ratio) / (1 + ratio), x, x2;
            r0 = r0 * r0;
            x = 1 - cos_theta;
            x2 = x * x;
            refl = r0 + (1 - r0) * x2 * x2 * x > rng_real(r);
        }
        *dir = refl ? reflect(unit, rec->normal) : refract(unit, rec->normal, ratio);
        return 1;
    }
    return 0; /* diffuse_light :101 */
}

/* ---- the integrator (renderer.hpp) ------------------------------------------------- */
static v3 background(const po_scene* s, v3 d) { /* :24-29 */
    v3 unit;
    float t;
    if (!s->d.sky) return mk(0, 0, 0);
    unit = normalize(d);
    t = 0.5f * (unit.y + 1);
    return add(scl(mk(1, 1, 1), 1 - t), scl(mk(0.5f, 0.7f, 1.0f), t));
}

static v3 direct_light(const po_scene* s, const rec_t* rec, const sampler_t* q, rng_t* r, uint64_t* rays,
                       counts* cnt) { /* :41-80 */
    uint32_t n = s->n_lights, pick;
    const pt_sphere* L;
    v3 to_center, w, a, u, v, dir, pl, outward;
    float dist2, r2, sin2_max, cos_max, omc, s1, s2, cos_t, sin_t, phi, cos_surface, t_light, pdf;
    pick = (uint32_t)(rng_real(r) * (float)n);
    if (pick > n - 1) pick = n - 1;
    L = &s->d.spheres[s->lights[pick]];
    to_center = sub(ld3(L->center), rec->p);
    dist2 = dot(to_center, to_center);
    r2 = L->radius * L->radius;
    if (dist2 <= r2) return mk(0, 0, 0);
    sin2_max = r2 / dist2;
    cos_max = sqrtf(1 - sin2_max);
    omc = sin2_max / (1 + cos_max);
    w = vdiv(to_center, sqrtf(dist2));
    a = fabsf(w.x) > 0.9f ? mk(0, 1, 0) : mk(1, 0, 0);
    u = normalize(cross(w, a));
    v = cross(w, u);
    sample_2d(q, r, 1, &s1, &s2);
    cos_t = 1 - s1 * omc;
    sin_t = sqrtf(fmaxf(0.0f, 1 - cos_t * cos_t));
    phi = 2 * (float)M_PI * s2;
    dir = add(add(scl(u, cosf(phi) * sin_t), scl(v, sinf(phi) * sin_t)), scl(w, cos_t));
    cos_surface = dot(dir, rec->normal);
    if (cos_surface <= 0) return mk(0, 0, 0);
    t_light = INFINITY;
    if (!sphere_hit(L, rec->p, dir, 0.001f, &t_light)) return mk(0, 0, 0);
    ++*rays;
    if (occluded(s, rec->p, dir, 0.001f, t_light * 0.9999f, cnt)) return mk(0, 0, 0);
    pl = add(rec->p, scl(dir, t_light));
    outward = scl(sub(pl, ld3(L->center)), 1 / L->radius);
    if (!(dot(dir, outward) < 0)) return mk(0, 0, 0);
    pdf = 1 / (2 * (float)M_PI * omc);
    return scl(ld3(s->d.materials[L->material].emission), cos_surface / (float)M_PI / pdf * (float)n);
}

/* ---- extended light sampling (PT_FLAG_NEE_EXTENDED; beyond the reference) ----------- */
/* The density of metal's scattered direction (material.hpp:85-91: mirror r
 * plus fuzz f times a point uniform in the unit ball) per unit solid angle at
 * unit direction w: over the chord [t1, t2] of the ray t*w (t >= 0) through
 * the ball of radius f about r, (t2^3 - t1^3) / (4 pi f^3). */
static float metal_lobe_pdf(v3 rr, float f, v3 w) {
    const float b = dot(w, rr), c = dot(rr, rr) - f * f;
    const float disc = b * b - c;
    float sq, t1, t2;
    if (!(disc > 0)) return 0;
    sq = sqrtf(disc);
    t2 = b + sq;
    if (!(t2 > 0)) return 0;
    t1 = fmaxf(b - sq, 0.0f);
    return (t2 * t2 * t2 - t1 * t1 * t1) / (4 * (float)M_PI * (f * f * f));
}
float po_metal_lobe_pdf(const float r[3], float f, const float w[3]) { return metal_lobe_pdf(ld3(r), f, ld3(w)); }

static uint32_t pick_light_ext(const po_scene* s, float u) {
    uint32_t lo = 0, hi = s->n_lights + s->n_tri_lights - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (u < s->light_cdf[mid]) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

/* A light sample of the extended list from rec: the matte estimate
 * (albedo / pi times the cosine; the albedo applied by the caller) or, with
 * metal, the lobe density weighted against the scattered ray by the power
 * heuristic. */
static v3 direct_light_ext(const po_scene* s, const rec_t* rec, v3 mirror, float fuzz, int metal, const sampler_t* q,
                           rng_t* r, uint64_t* rays, counts* cnt) {
    const uint32_t k = pick_light_ext(s, rng_real(r));
    v3 dir, le;
    float cos_surface, pdf_solid, power, t_max, pdf, f, s1, s2;
    int front = 1;
    if (k < s->n_lights) {
        const pt_sphere* L = &s->d.spheres[s->lights[k]];
        v3 to_center, w, a, u, v, outward;
        float dist2, r2, sin2_max, cos_max, omc, cos_t, sin_t, phi, t_light;
        to_center = sub(ld3(L->center), rec->p);
        dist2 = dot(to_center, to_center);
        r2 = L->radius * L->radius;
        if (dist2 <= r2) return mk(0, 0, 0);
        sin2_max = r2 / dist2;
        cos_max = sqrtf(1 - sin2_max);
        omc = sin2_max / (1 + cos_max);
        w = vdiv(to_center, sqrtf(dist2));
        a = fabsf(w.x) > 0.9f ? mk(0, 1, 0) : mk(1, 0, 0);
        u = normalize(cross(w, a));
        v = cross(w, u);
        sample_2d(q, r, 1, &s1, &s2);
        cos_t = 1 - s1 * omc;
        sin_t = sqrtf(fmaxf(0.0f, 1 - cos_t * cos_t));
        phi = 2 * (float)M_PI * s2;
        dir = add(add(scl(u, cosf(phi) * sin_t), scl(v, sinf(phi) * sin_t)), scl(w, cos_t));
        cos_surface = dot(dir, rec->normal);
        if (cos_surface <= 0) return mk(0, 0, 0);
        t_light = INFINITY;
        if (!sphere_hit(L, rec->p, dir, 0.001f, &t_light)) return mk(0, 0, 0);
        ++*rays;
        outward = scl(sub(add(rec->p, scl(dir, t_light)), ld3(L->center)), 1 / L->radius);
        front = dot(dir, outward) < 0;
        t_max = t_light * 0.9999f;
        pdf_solid = 1 / (2 * (float)M_PI * omc);
        le = ld3(s->d.materials[L->material].emission);
        power = sphere_power(light_lum(s->d.materials[L->material].emission), L->radius);
    } else {
        const uint32_t ti = k - s->n_lights;
        const pt_triangle* T = &s->d.triangles[s->tri_lights[ti]];
        const float area = s->tri_area[ti];
        float sq, dist2, dist, cos_l;
        v3 y, dv;
        sample_2d(q, r, 1, &s1, &s2);
        sq = sqrtf(s1);
        y = add(add(ld3(T->p0), scl(ld3(T->e1), 1 - sq)), scl(ld3(T->e2), s2 * sq));
        dv = sub(y, rec->p);
        dist2 = dot(dv, dv);
        if (!(dist2 > 0)) return mk(0, 0, 0);
        dist = sqrtf(dist2);
        dir = scl(dv, 1.0f / dist);
        cos_l = -dot(dir, ld3(T->face_normal));
        if (!(cos_l > 0)) return mk(0, 0, 0);
        cos_surface = dot(dir, rec->normal);
        if (cos_surface <= 0) return mk(0, 0, 0);
        ++*rays;
        t_max = dist * 0.9999f;
        pdf_solid = dist2 / (area * cos_l);
        le = ld3(s->d.materials[T->material].emission);
        power = tri_power(light_lum(s->d.materials[T->material].emission), area);
    }
    pdf = (s->pick_uniform + s->pick_power * power) * pdf_solid;
    if (!(pdf > 0) || !(pdf < 3.0e38f)) return mk(0, 0, 0);
    if (metal) {
        const float pb = metal_lobe_pdf(mirror, fuzz, dir), qq = pb / pdf;
        f = qq * (1 / (1 + qq * qq));
    } else {
        f = cos_surface / (float)M_PI / pdf;
    }
    if (!front || !(f > 0)) return mk(0, 0, 0);
    if (occluded(s, rec->p, dir, 0.001f, t_max, cnt)) return mk(0, 0, 0);
    return scl(le, f);
}

/* The extended light-sampling density of direction d from x that hit the light in rec. */
static float light_pdf_at_hit(const po_scene* s, const rec_t* rec, v3 x, v3 d, const float* em) {
    float pdf_solid, power;
    const float lum = light_lum(em);
    if (rec->lkind == 1) {
        const v3 to_center = sub(rec->lgeo, x);
        const float dist2 = dot(to_center, to_center), r2 = rec->lw * rec->lw;
        float sin2_max;
        if (dist2 <= r2) return 0;
        sin2_max = r2 / dist2;
        pdf_solid = 1 / (2 * (float)M_PI * (sin2_max / (1 + sqrtf(1 - sin2_max))));
        power = sphere_power(lum, rec->lw);
    } else {
        const float dl = sqrtf(dot(d, d)), dist = rec->t * dl;
        const float cos_l = fabsf(dot(d, rec->lgeo)) / dl;
        pdf_solid = dist * dist / (rec->lw * cos_l);
        power = tri_power(lum, rec->lw);
    }
    return (s->pick_uniform + s->pick_power * power) * pdf_solid;
}

/* ray_color<with_first> (:100-149); ext: the extended light sampling. */
static v3 ray_color(const po_scene* s, v3 o, v3 d, int depth, sampler_t* q, rng_t* r, v3* f_albedo, v3* f_normal,
                    uint64_t* rays, counts* cnt, int ext) {
    v3 tp = mk(1, 1, 1), rad = mk(0, 0, 0);
    int sampled = 0, bounce;
    float mis_pdf = 0;
    for (bounce = 0; bounce < depth; ++bounce) {
        rec_t rec;
        const pt_material* m;
        v3 att, dir;
        int scatters;
        ++*rays;
        q->base = 1 + 2 * bounce;
        if (!hit(s, o, d, 0.001f, 1000, &rec, cnt, ext)) {
            if (bounce == 0) {
                *f_albedo = mk(1, 1, 1);
                *f_normal = mk(0, 0, 0);
            }
            return add(rad, mul(tp, background(s, d)));
        }
        m = &s->d.materials[rec.mat];
        if (rec.front_face && !(sampled && rec.sampled_light)) {
            if (ext && mis_pdf > 0 && rec.sampled_light) {
                const float qq = light_pdf_at_hit(s, &rec, o, d, m->emission) / mis_pdf;
                rad = add(rad, mul(tp, scl(ld3(m->emission), 1 / (1 + qq * qq))));
            } else {
                rad = add(rad, mul(tp, ld3(m->emission)));
            }
        }
        scatters = scatter(m, d, &rec, q, r, &att, &dir);
        /* lambertian: albedo * texture->sample(tex_u, tex_v) (material.hpp:72) */
        if (m->type == PT_MAT_LAMBERTIAN && m->texture > 0) att = mul(att, sample_texture(s, m->texture - 1, rec.tex_u, rec.tex_v));
        if (bounce == 0) {
            *f_albedo = scatters && m->type != PT_MAT_DIELECTRIC ? att : mk(1, 1, 1);
            *f_normal = rec.normal;
        }
        if (ext) {
            const int can = s->d.sample_lights && s->n_lights + s->n_tri_lights > 0 && bounce + 1 < depth;
            const float fuzz = m->fuzz < 1 ? m->fuzz : 1;
            mis_pdf = 0;
            if (m->type == PT_MAT_METAL && fuzz > 1e-3f && can) {
                const v3 mirror = reflect(normalize(d), rec.normal);
                rad = add(rad, mul(mul(tp, att), direct_light_ext(s, &rec, mirror, fuzz, 1, q, r, rays, cnt)));
                if (scatters) mis_pdf = metal_lobe_pdf(mirror, fuzz, normalize(dir));
            }
            if (!scatters) return rad;
            sampled = m->type == PT_MAT_LAMBERTIAN && can;
            if (sampled) rad = add(rad, mul(mul(tp, att), direct_light_ext(s, &rec, mk(0, 0, 0), 0, 0, q, r, rays, cnt)));
        } else {
            if (!scatters) return rad;
            sampled = m->type == PT_MAT_LAMBERTIAN && s->d.sample_lights && s->n_lights > 0 && bounce + 1 < depth;
            if (sampled) rad = add(rad, mul(mul(tp, att), direct_light(s, &rec, q, r, rays, cnt)));
        }
        tp = mul(tp, att);
        o = rec.p;
        d = dir;
        if (bounce + 1 >= 3) {
            float p = fmaxf(tp.x, fmaxf(tp.y, tp.z));
            if (p < 1) {
                if (rng_real(r) >= p) return rad;
                tp = vdiv(tp, p);
            }
        }
    }
    return rad;
}

static float luminance(v3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; } /* :364 */

/*
 * Renders scanlines [row0, row0 + rows) of a W x H image in the layout of
 * pt_render (3 floats per pixel, top row first; aux 7 floats or NULL).
 * rng_mode: 0 = per-(pixel, sample) streams (PT_RNG_SAMPLE), 1 = caller's
 * per-sample states (PT_RNG_SNAPSHOT), 2 = the reference's own per-row stream
 * (seed_row, renderer.hpp:349-351). render_row_impl (:366-409).
 */
void po_render_flags(const po_scene* s, const pt_camera* cam, int W, int H, int spp, int depth, uint64_t seed,
                     int first_sample, int rng_mode, const uint64_t* states, int row0, int rows, float* out,
                     float* aux, uint64_t* rays_out, uint64_t counts_out[5], int flags) {
    v3 origin = ld3(cam->origin), llc = ld3(cam->lower_left), hz = ld3(cam->horizontal), vt = ld3(cam->vertical);
    float scale = 1.0f / spp;
    uint64_t rays = 0;
    counts cnt;
    int j;
    sobol_init();
    memset(&cnt, 0, sizeof(cnt));
    for (j = row0; j < row0 + rows; ++j) {
        rng_t r;
        int i;
        if (rng_mode == 2) rng_seed(&r, seed ^ (((uint64_t)(uint32_t)j << 32) | (uint32_t)first_sample));
        for (i = 0; i < W; ++i) {
            v3 pc = mk(0, 0, 0), alb = mk(0, 0, 0), nor = mk(0, 0, 0);
            float lum2 = 0;
            size_t px = (size_t)(H - 1 - j) * W + i;
            int k;
            for (k = 0; k < spp; ++k) {
                sampler_t q;
                float du, dv, u, v;
                v3 dir, c, fa = mk(0, 0, 0), fn = mk(0, 0, 0);
                uint32_t idx = (uint32_t)(first_sample + k);
                begin_sample(&q, seed, i, j, idx);
                sample_2d(&q, &r, 0, &du, &dv);
                u = ((float)i + du) / (float)(W - 1);
                v = ((float)j + dv) / (float)(H - 1);
                dir = sub(add(add(llc, scl(hz, u)), scl(vt, v)), origin);
                if (rng_mode == 0) rng_seed(&r, po_sample_stream_seed(seed, i, j, idx));
                if (rng_mode == 1) memcpy(r.s, states + 4 * (((size_t)j * W + i) * spp + k), 32);
                c = ray_color(s, origin, dir, depth, &q, &r, &fa, &fn, &rays, counts_out ? &cnt : NULL,
                              (flags & PT_FLAG_NEE_EXTENDED) != 0);
                pc = add(pc, c);
                alb = add(alb, fa);
                nor = add(nor, fn);
                lum2 += luminance(c) * luminance(c);
            }
            out[3 * px] = pc.x * scale;
            out[3 * px + 1] = pc.y * scale;
            out[3 * px + 2] = pc.z * scale;
            if (aux) {
                float* a = aux + 7 * px;
                a[0] = alb.x * scale;
                a[1] = alb.y * scale;
                a[2] = alb.z * scale;
                a[3] = nor.x * scale;
                a[4] = nor.y * scale;
                a[5] = nor.z * scale;
                a[6] = lum2 * scale;
            }
        }
    }
    if (rays_out) *rays_out = rays;
    if (counts_out) {
        counts_out[0] = cnt.nodes;
        counts_out[1] = cnt.order;
        counts_out[2] = cnt.tris;
        counts_out[3] = cnt.spheres;
        counts_out[4] = cnt.insts;
    }
}

void po_render(const po_scene* s, const pt_camera* cam, int W, int H, int spp, int depth, uint64_t seed,
               int first_sample, int rng_mode, const uint64_t* states, int row0, int rows, float* out, float* aux,
               uint64_t* rays_out, uint64_t counts_out[5]) {
    po_render_flags(s, cam, W, H, spp, depth, seed, first_sample, rng_mode, states, row0, rows, out, aux, rays_out,
                    counts_out, 0);
}

/* Ray queries: geometry::hit's choice and geometry::occluded, per ray. */
void po_trace_closest(const po_scene* s, const float* rays, size_t n, float tmin, float tmax, pt_hit* out,
                      uint64_t counts_out[5]) {
    counts cnt;
    size_t i;
    memset(&cnt, 0, sizeof(cnt));
    for (i = 0; i < n; ++i) {
        const float* r = rays + 6 * i;
        hctx c;
        float t = tmax;
        closest(s, mk(r[0], r[1], r[2]), mk(r[3], r[4], r[5]), tmin, &t, &c, counts_out ? &cnt : NULL);
        out[i].kind = c.kind;
        out[i].index = c.kind == PT_HIT_NONE ? 0 : c.index;
        out[i].sub = c.kind == PT_HIT_INSTANCE ? c.sub : 0;
        out[i].t = t;
        out[i].u = c.u;
        out[i].v = c.v;
    }
    if (counts_out) {
        counts_out[0] = cnt.nodes;
        counts_out[1] = cnt.order;
        counts_out[2] = cnt.tris;
        counts_out[3] = cnt.spheres;
        counts_out[4] = cnt.insts;
    }
}

void po_trace_any(const po_scene* s, const float* rays, size_t n, float tmin, float tmax, uint8_t* out) {
    size_t i;
    for (i = 0; i < n; ++i) {
        const float* r = rays + 6 * i;
        out[i] = (uint8_t)occluded(s, mk(r[0], r[1], r[2]), mk(r[3], r[4], r[5]), tmin, tmax, NULL);
    }
}

/* The a-trous denoiser (denoise.hpp:55-139), single-threaded. */
static float lumf(const float* c) { return 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]; }

void po_denoise(int w, int h, const float* color, const float* albedo, const float* normal, const float* variance,
                float* out) {
    const float kernel[3] = {3.0f / 8, 1.0f / 4, 1.0f / 16};
    const float sigma_l = 4, albedo_sigma2 = 0.01f;
    size_t n = (size_t)w * h, p;
    float *light = (float*)malloc(3 * n * sizeof(float)), *light_next = (float*)malloc(3 * n * sizeof(float));
    float *var = (float*)malloc(n * sizeof(float)), *var_next = (float*)malloc(n * sizeof(float));
    float* nrm = (float*)malloc(3 * n * sizeof(float));
    int pass, c;
    for (p = 0; p < n; ++p) {
        float a, len;
        const float* sn = normal + 3 * p;
        for (c = 0; c < 3; ++c) light[3 * p + c] = color[3 * p + c] / fmaxf(albedo[3 * p + c], 0.01f);
        a = fmaxf(lumf(albedo + 3 * p), 0.01f);
        var[p] = fmaxf(variance[p], 0.0f) / (a * a);
        len = sqrtf(sn[0] * sn[0] + sn[1] * sn[1] + sn[2] * sn[2]);
        for (c = 0; c < 3; ++c) nrm[3 * p + c] = len > 1e-6f ? sn[c] / len : 0;
    }
    for (pass = 0; pass < 5; ++pass) {
        int step = 1 << pass, x, y;
        float* tmp;
        for (y = 0; y < h; ++y)
            for (x = 0; x < w; ++x) {
                size_t pp = (size_t)y * w + x;
                const float* np = &nrm[3 * pp];
                const float* ap = albedo + 3 * pp;
                int p_sky = np[0] == 0 && np[1] == 0 && np[2] == 0, dx, dy;
                float lp = lumf(&light[3 * pp]), v = 0, vw = 0, sc, sum[3] = {0, 0, 0}, sum_w = 0, sum_var = 0;
                for (dy = -1; dy <= 1; ++dy)
                    for (dx = -1; dx <= 1; ++dx) {
                        int qx = x + dx, qy = y + dy;
                        float k;
                        if (qx < 0 || qy < 0 || qx >= w || qy >= h) continue;
                        k = (dx ? 0.5f : 1) * (dy ? 0.5f : 1);
                        v += k * var[(size_t)qy * w + qx];
                        vw += k;
                    }
                sc = 1 / (sigma_l * sqrtf(v / vw) + 1e-4f);
                for (dy = -2; dy <= 2; ++dy) {
                    int qy = y + dy * step;
                    if (qy < 0 || qy >= h) continue;
                    for (dx = -2; dx <= 2; ++dx) {
                        int qx = x + dx * step, q_sky, k;
                        size_t q;
                        const float *nq, *aq;
                        float weight, da0, da1, da2;
                        if (qx < 0 || qx >= w) continue;
                        q = (size_t)qy * w + qx;
                        nq = &nrm[3 * q];
                        aq = albedo + 3 * q;
                        q_sky = nq[0] == 0 && nq[1] == 0 && nq[2] == 0;
                        if (p_sky != q_sky) continue;
                        weight = kernel[abs(dx)] * kernel[abs(dy)];
                        if (!p_sky) {
                            float nd = fmaxf(np[0] * nq[0] + np[1] * nq[1] + np[2] * nq[2], 0.0f);
                            for (k = 0; k < 6; ++k) nd *= nd;
                            weight *= nd;
                        }
                        da0 = ap[0] - aq[0];
                        da1 = ap[1] - aq[1];
                        da2 = ap[2] - aq[2];
                        weight *= expf(-(da0 * da0 + da1 * da1 + da2 * da2) * (1 / albedo_sigma2) -
                                       fabsf(lp - lumf(&light[3 * q])) * sc);
                        for (c = 0; c < 3; ++c) sum[c] += weight * light[3 * q + c];
                        sum_w += weight;
                        sum_var += weight * weight * var[q];
                    }
                }
                for (c = 0; c < 3; ++c) light_next[3 * pp + c] = sum[c] / sum_w;
                var_next[pp] = sum_var / (sum_w * sum_w);
            }
        tmp = light;
        light = light_next;
        light_next = tmp;
        tmp = var;
        var = var_next;
        var_next = tmp;
    }
    for (p = 0; p < n; ++p)
        for (c = 0; c < 3; ++c) out[3 * p + c] = light[3 * p + c] * fmaxf(albedo[3 * p + c], 0.01f);
    free(light);
    free(light_next);
    free(var);
    free(var_next);
    free(nrm);
}
