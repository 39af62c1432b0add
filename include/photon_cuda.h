/*
 * photon_cuda.h -- C ABI of the B200 (sm_100a) render hot path of photon_tracer.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns a pt_status; no C++ exception and no torch type crosses it. A
 * caller that builds its scene with photon_tracer's `geometry`/`camera` API
 * converts it with the header-only shim photon_cuda_geometry.hpp and then
 * renders through pt_render / pt_render_row in place of the CPU call.
 *
 * Each declaration names the reference interface it replaces
 * (photon_tracer file:line). Layouts that must match the reference byte for
 * byte (pt_bvh_node) say so.
 *
 * Threading: a pt_scene owns one CUDA stream for the host-buffer entry
 * points. Calls on one handle must be serialised by the caller; different
 * handles may be used from different threads. pt_last_error() is per thread.
 */
#ifndef PHOTON_CUDA_H
#define PHOTON_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PT_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
/* Replaces the reference's std::runtime_error / exit codes
 * (include/gpu_pack.hpp:62,86; src/main.cpp:58-61,103-108). */
typedef int32_t pt_status;
enum {
    PT_OK = 0,
    PT_ERR_INVALID_ARG = 1,     /* null pointer, bad size, index out of range */
    PT_ERR_OUT_OF_MEMORY = 2,   /* device or host allocation failed */
    PT_ERR_STACK_OVERFLOW = 3,  /* a traversal stack would overflow (scene refused or ray flagged) */
    PT_ERR_QUEUE_OVERFLOW = 4,  /* a wavefront queue overflowed */
    PT_ERR_TIMEOUT = 5,         /* a bounded device wait ran out */
    PT_ERR_CUDA = 6,            /* a CUDA runtime call failed; pt_last_error() has the text */
    PT_ERR_NO_DEVICE = 7,       /* no CUDA device, or not sm_100 */
    PT_ERR_UNSUPPORTED = 8      /* a feature combination the library does not implement */
};

/* Text of the last error on the calling thread ("" if none). */
const char* pt_last_error(void);
/* Library version string, e.g. "photon_cuda 0.1 (sm_100a)". */
const char* pt_version(void);

/* ---- scene description --------------------------------------------------- */
/* Material kinds: the reference's material subclasses (include/material.hpp:46-137),
 * mapped the way include/gpu_pack.hpp:89-113 maps them (lambertian 0, metal 1,
 * dielectric 2, anything else a light, 3). */
enum { PT_MAT_LAMBERTIAN = 0, PT_MAT_METAL = 1, PT_MAT_DIELECTRIC = 2, PT_MAT_DIFFUSE_LIGHT = 3 };
#define PT_NO_MATERIAL 0xffffffffu

/* One material: include/material.hpp:13-30 (emission, diffuse, transmissive)
 * plus the subclass fields (albedo :48, fuzz :81 -- the library applies the
 * metal constructor's clamp f < 1 ? f : 1 (:83) --, ior :109).
 * diffuse/transmissive follow from type. */
typedef struct pt_material {
    uint32_t type;
    float albedo[3];
    float emission[3];
    float fuzz;
    float ior;
    uint32_t texture; /* lambertian::texture (:50): 0 for none, k for pt_scene_desc.textures[k - 1]
                         (so a zeroed material has none); the albedo is then multiplied by the
                         texture at the hit's texture coordinates */
} pt_material;

/* An image texture (include/texture.hpp:9-48): width x height texels of sRGB
 * bytes, 3 per texel, rows top first (the image8 the reference decodes). */
typedef struct pt_texture {
    int32_t width, height;
    const uint8_t* rgb;
} pt_texture;

/* A sphere: include/sphere.hpp:15-17. A negative radius is a hollow shell. */
typedef struct pt_sphere {
    float center[3];
    float radius;
    uint32_t material;
} pt_sphere;

/* A triangle, the fields include/triangle.hpp:14-24 stores, as the
 * reference's constructor computed them (e1 = p1 - p0, e2 = p2 - p0,
 * face_normal = normalize(cross(e1, e2)); vertex normals = face normal for
 * a flat triangle). p1 and p2 are the corners as given, which the bounding
 * box (include/triangle.hpp:76-83) is taken from. uv holds the texture
 * coordinates at the three corners. pt_triangle_init fills the derived
 * fields the reference's way. */
typedef struct pt_triangle {
    float p0[3], e1[3], e2[3];
    float n0[3], n1[3], n2[3];
    float face_normal[3];
    float p1[3], p2[3];
    uint32_t material;
    float uv[6];  /* texture coordinates at the three corners (include/triangle.hpp:20) */
} pt_triangle;

/* A 3x3 + translation affine transform: include/transform.hpp:11-12. */
typedef struct pt_affine {
    float m[3][3];
    float t[3];
} pt_affine;

/* One 4-wide BVH node, byte for byte the reference's bvh::node
 * (include/bvh.hpp:27-32): child c is a leaf when count[c] > 0 (primitives
 * order[first[c], first[c] + count[c])), an interior node nodes[first[c]]
 * otherwise; unused slots have boxes at +infinity. */
typedef struct pt_bvh_node {
    float lo[3][4];
    float hi[3][4];
    uint32_t first[4];
    uint32_t count[4];
} pt_bvh_node;

/* A built tree: bvh::nodes and bvh::order (include/bvh.hpp:35-36). */
typedef struct pt_bvh {
    const pt_bvh_node* nodes;
    uint32_t n_nodes;
    const uint32_t* order;
    uint32_t n_order;
} pt_bvh;

/* A mesh for instancing: geometry::mesh (include/geometry.hpp:47-51). With
 * tree.nodes NULL the library builds the tree with its own builder, which
 * produces the same nodes and order as bvh::build (include/bvh.hpp:39-52). */
typedef struct pt_mesh {
    const pt_triangle* triangles;
    uint32_t n_triangles;
    pt_bvh tree;
} pt_mesh;

/* An instance: geometry::instance (include/geometry.hpp:52-56). to_object is
 * the inverse of to_world as affine::inverse (include/transform.hpp:42-59)
 * computed it; material PT_NO_MATERIAL keeps the mesh's own materials. */
typedef struct pt_instance {
    uint32_t mesh;
    uint32_t material;
    pt_affine to_world;
    pt_affine to_object;
} pt_instance;

/* Everything class geometry holds (include/geometry.hpp:15-58, 193-195).
 * Trees given as NULL are built by the library (when use_bvh); trees given
 * must be the ones the reference built for this geometry. lights NULL means
 * "derive them as geometry::build does" (emissive spheres, :75-77). */
typedef struct pt_scene_desc {
    const pt_material* materials;
    uint32_t n_materials;
    const pt_sphere* spheres;
    uint32_t n_spheres;
    const pt_sphere* large_spheres;
    uint32_t n_large_spheres;
    const pt_triangle* triangles;
    uint32_t n_triangles;
    const pt_mesh* meshes;
    uint32_t n_meshes;
    const pt_instance* instances;
    uint32_t n_instances;
    pt_bvh flat_tree;
    pt_bvh instance_tree;
    const uint32_t* lights;
    uint32_t n_lights;
    int32_t sky;           /* geometry::sky (:30) */
    int32_t sample_lights; /* geometry::sample_lights (:32), next event estimation */
    int32_t use_bvh;       /* geometry::build(use_bvh) (:74) */
    const pt_texture* textures; /* the images textured lambertians refer to */
    uint32_t n_textures;
} pt_scene_desc;

typedef struct pt_scene pt_scene;

/* Sizes of what pt_scene_create put on the device. */
typedef struct pt_scene_info {
    uint32_t n_nodes;       /* 4-wide nodes over all trees */
    uint32_t n_slots;       /* leaf slots over all trees */
    uint32_t max_depth;     /* deepest 4-wide tree (levels) */
    uint32_t stack_entries; /* traversal stack entries a ray can need */
    uint64_t device_bytes;  /* device memory the scene holds */
} pt_scene_info;

/* Deep-copies desc to device memory (the caller keeps its buffers) and
 * repacks every tree into one node arena. Replaces the scene hand-off of
 * include/gpu_pack.hpp:84-175 (pack_for_gpu). */
pt_status pt_scene_create(const pt_scene_desc* desc, pt_scene** out);
pt_status pt_scene_destroy(pt_scene* scene);
pt_status pt_scene_get_info(const pt_scene* scene, pt_scene_info* info);

/* ---- camera -------------------------------------------------------------- */
/* class camera's four fields (include/camera.hpp:10-13, accessors :39-42). */
typedef struct pt_camera {
    float origin[3];
    float lower_left[3];
    float horizontal[3];
    float vertical[3];
} pt_camera;

/* camera(lookfrom, lookat, vfov_deg) (include/camera.hpp:18-34) with the
 * aspect ratio as a parameter; aspect 16/9 gives the reference's camera
 * bit for bit. */
pt_status pt_camera_look_at(const float lookfrom[3], const float lookat[3], double vfov_deg, double aspect,
                            pt_camera* out);

/* ---- rendering ------------------------------------------------------------ */
enum { PT_MODE_AUTO = 0, PT_MODE_MEGAKERNEL = 1, PT_MODE_WAVEFRONT = 2 };
/* Random streams. PT_RNG_SAMPLE: one xoshiro256+ stream per (pixel, sample),
 * seeded from (seed, pixel, sample) -- order independent, the production
 * mode. PT_RNG_SNAPSHOT: the caller supplies each sample's starting
 * xoshiro256+ state (4 words, sample-major within a pixel, pixels row by
 * row from the bottom row j = 0), e.g. captured from the reference's own
 * per-row stream (src/main.cpp:150 -> include/renderer.hpp:349-351). */
enum { PT_RNG_SAMPLE = 0, PT_RNG_SNAPSHOT = 1 };

/* Flags of pt_settings. 0 renders exactly the reference's estimator.
 *
 * PT_FLAG_NEE_EXTENDED -- beyond the reference, which names both as known
 * limits (README.md:453-456): next-event estimation toward emissive
 * triangles, and from rough metal. With it:
 *   - the light list is every emissive light sphere (as the reference's) plus
 *     every emissive triangle of the flat triangle list (not those inside
 *     meshes placed by instances); a light is picked with probability
 *     proportional to its power (luminance of the emission times its area)
 *     instead of uniformly among spheres;
 *   - a light sphere is sampled over its cone as include/renderer.hpp:41-80
 *     does, a triangle uniformly over its area; matte surfaces use these
 *     samples as the reference does (light hit afterwards not counted again);
 *   - metal with fuzz above 1e-3 also samples a light and weights that sample
 *     and its own scattered ray by the power heuristic (multiple importance
 *     sampling), with the exact density of its fuzz-ball lobe;
 *   - glass and fuzz-0 metal reflect or refract into one direction only, so
 *     no light sample can reach them: their light still arrives through
 *     their scattered rays, as in the reference.
 * It renders with the megakernel and production streams: with
 * PT_MODE_WAVEFRONT or PT_RNG_SNAPSHOT the call fails with PT_ERR_UNSUPPORTED.
 * Batches and the row call (pt_render_row) render without it. */
enum { PT_FLAG_NEE_EXTENDED = 1 };

typedef struct pt_settings {
    int32_t width, height;
    int32_t spp;          /* samples_per_pixel */
    int32_t max_bounces;  /* depth, 10 in src/main.cpp:84 */
    uint64_t seed;
    int32_t first_sample; /* progressive continuation, include/renderer.hpp:411-413 */
    int32_t mode;         /* PT_MODE_* */
    int32_t rng;          /* PT_RNG_* */
    int32_t flags;        /* PT_FLAG_*; 0: the reference's estimator */
    const uint64_t* rng_states; /* PT_RNG_SNAPSHOT only: width*height*spp*4 words */
} pt_settings;

/* Progressive rendering (the web front end's render loop, web/gpu.js:205-226):
 * the frame's samples in batches that start at 1 spp and double while a batch
 * takes under 20 ms (up to 64) or halve above 60 ms, each batch continuing
 * the per-pixel sample numbering (first_sample + samples done), its averages
 * summed per pixel in FP64. After each batch but the last, progress (may be
 * NULL) is called with the samples done so far; a nonzero return stops the
 * render there. out (host, 3 floats per pixel, top row first) gets the mean
 * of the samples done, *samples_done (may be NULL) their count. Needs
 * PT_RNG_SAMPLE; no aux. */
typedef int (*pt_progress_fn)(void* user, int32_t samples_done, int32_t samples_total);
pt_status pt_render_progressive(pt_scene* scene, const pt_camera* cam, const pt_settings* settings, float* out,
                                pt_progress_fn progress, void* user, int32_t* samples_done, uint64_t* rays_out);

/* Renders a frame. Replaces the per-row calls of
 * render_row_linear(world, cam, j, W, H, spp, depth, out, seed, first_sample, aux)
 * (include/renderer.hpp:411-416) over every row, in the layout
 * src/main.cpp:124-151 produces: out is 3*W*H floats, TOP row first (row
 * H-1-j holds scanline j); aux (NULL or 7*W*H floats) is the per-pixel
 * albedo(3), normal(3), mean squared luminance(1) of include/renderer.hpp:358-362.
 * rays_out (may be NULL) receives the ray count with the reference's
 * convention (include/renderer.hpp:72,110). Host buffers; blocks until done. */
pt_status pt_render(pt_scene* scene, const pt_camera* cam, const pt_settings* settings, float* out, float* aux,
                    uint64_t* rays_out);

/* The same with DEVICE buffers, enqueued on `stream` (a cudaStream_t, NULL
 * for the legacy default stream) without synchronising. d_rays (may be NULL)
 * is one device uint64 that the ray count is ADDED to. settings->rng_states
 * must be a device pointer. Kernel-side errors (stack overflow, timeouts)
 * are reported by the next pt_sync(). */
pt_status pt_render_device(pt_scene* scene, const pt_camera* cam, const pt_settings* settings, float* d_out,
                           float* d_aux, uint64_t* d_rays, void* stream);

/* One scanline: the exact signature and meaning of render_row_linear
 * (include/renderer.hpp:411-416); out is 3*width floats, aux NULL or
 * 7*width. Seeds the reference's way for row j (seed_row, :349-351) is not
 * reproduced: samples use PT_RNG_SAMPLE streams. Host buffers; blocking. */
pt_status pt_render_row(pt_scene* scene, const pt_camera* cam, int j, int width, int height, int samples_per_pixel,
                        int max_bounces, float* out, uint64_t seed, int first_sample, float* aux);

/* Waits for the scene's device work on `stream` and reports any error a
 * kernel flagged since the last call. */
pt_status pt_sync(pt_scene* scene, void* stream);

/* ---- ray queries ---------------------------------------------------------- */
/* What geometry::hit found (include/geometry.hpp:113-115): kind, index and
 * sub-triangle of the nearest primitive, its t and barycentrics. */
enum { PT_HIT_NONE = 0, PT_HIT_LARGE = 1, PT_HIT_SPHERE = 2, PT_HIT_TRIANGLE = 3, PT_HIT_INSTANCE = 4 };
typedef struct pt_hit {
    uint32_t kind;
    uint32_t index; /* large sphere, sphere, triangle or instance number */
    uint32_t sub;   /* triangle within the instanced mesh */
    float t, u, v;
} pt_hit;

/* Closest hit for n rays (6 floats each: origin, direction) in [tmin, tmax]:
 * geometry::hit (include/geometry.hpp:111-152), bit-exact. Host buffers. */
pt_status pt_trace_closest(pt_scene* scene, const float* rays, size_t n, float tmin, float tmax, pt_hit* hits);
/* Any hit: geometry::occluded (include/geometry.hpp:156-190); occluded[i] is 1 or 0. */
pt_status pt_trace_any(pt_scene* scene, const float* rays, size_t n, float tmin, float tmax, uint8_t* occluded);
/* Device-buffer forms, enqueued on stream. */
pt_status pt_trace_closest_device(pt_scene* scene, const float* d_rays, size_t n, float tmin, float tmax,
                                  pt_hit* d_hits, void* stream);
pt_status pt_trace_any_device(pt_scene* scene, const float* d_rays, size_t n, float tmin, float tmax,
                              uint8_t* d_occluded, void* stream);

/* Distance to the first surface along each pixel's centre ray (u = (i+0.5)/(W-1),
 * v = (j+0.5)/(H-1) on include/camera.hpp:39-47), width*height floats, top row
 * first, 0 where the ray leaves the scene: the depth guide of pt_denoise_unet.
 * No reference counterpart (the reference's guides are albedo and normal,
 * src/main.cpp:176-183). Device buffer, enqueued on stream. */
pt_status pt_primary_depth_device(pt_scene* scene, const pt_camera* cam, int width, int height, float* d_depth,
                                  void* stream);

/* Traversal work counters for the algorithmic-bytes roofline: per ray, the
 * nodes visited, leaf-order entries read, triangles and spheres tested and
 * instances entered, summed over n rays (closest hit). Same traversal as
 * pt_trace_closest. counts[5] = {nodes, order, triangles, spheres, instances}. */
pt_status pt_trace_count(pt_scene* scene, const float* rays, size_t n, float tmin, float tmax, uint64_t counts[5]);

/* ---- triangles (host) ------------------------------------------------------ */
/* The reference's triangle constructors (include/triangle.hpp:26-35): e1, e2
 * and the face normal from the corners p0, p1, p2 in its float arithmetic;
 * normals (9 floats: n0, n1, n2) or, when null, the face normal at every
 * vertex (the flat constructor); texture coordinates zero. */
pt_status pt_triangle_init(const float p0[3], const float p1[3], const float p2[3], const float* normals,
                           uint32_t material, pt_triangle* out);

/* ---- instance transforms (host) -------------------------------------------- */
/* affine::inverse (include/transform.hpp:42-59): cofactors and determinant in
 * double, the linear part rounded to float, t = -(M^-1 t) in float. This is the
 * to_object a pt_instance must carry for its to_world. A singular to_world
 * gives infinite or NaN entries, as in the reference. */
pt_status pt_affine_inverse(const pt_affine* to_world, pt_affine* to_object);

/* ---- BVH build (host) ------------------------------------------------------ */
/* The library's own host builder: binned SAH (16 bins, leaf <= 8, depth <= 64)
 * collapsed to 4-wide nodes, producing the same nodes and order as
 * bvh::build (include/bvh.hpp:39-52, 126-247). boxes is n*6 floats (min xyz,
 * max xyz). Free the results with pt_free. */
pt_status pt_bvh_build(const float* boxes, uint32_t n, pt_bvh_node** nodes, uint32_t* n_nodes, uint32_t** order);
/* The same build on the GPU (binned SAH over primitive chunks for large
 * nodes, one thread per subtree of <= 128 primitives, the 4-wide collapse on
 * the host): the same nodes and order as pt_bvh_build, byte for byte, for
 * the same boxes (bvh::build, include/bvh.hpp:39-52, 126-247; the reference
 * builds on the host only). Host arrays in and out; free with pt_free. */
pt_status pt_bvh_build_gpu(const float* boxes, uint32_t n, pt_bvh_node** nodes, uint32_t* n_nodes, uint32_t** order);
void pt_free(void* p);

/* ---- denoising -------------------------------------------------------------- */
/* The edge-avoiding a-trous filter of include/denoise.hpp:55-139 on the GPU.
 * color/albedo/normal are 3 floats per pixel, variance 1; out 3. Host
 * buffers; blocking. Rows in any order as long as all inputs agree. */
pt_status pt_denoise_atrous(int width, int height, const float* color, const float* albedo, const float* normal,
                            const float* variance, float* out);
pt_status pt_denoise_atrous_device(int width, int height, const float* d_color, const float* d_albedo,
                                   const float* d_normal, const float* d_variance, float* d_out, float* d_scratch,
                                   void* stream);
/* Scratch floats pt_denoise_atrous_device needs for a width x height frame. */
size_t pt_denoise_atrous_scratch_floats(int width, int height);

/* No counterpart in the reference. The filter of pt_denoise_atrous_device for
 * callers that cannot allocate device memory (a host that owns all device
 * memory through its own pool, a frame loop where cudaMalloc -- which can
 * synchronise and can fail -- is not allowed): it calls no allocator and
 * takes its scratch from a fixed array inside the library, which every GPU
 * that loads the library holds (11.5 MB) until the process exits. Frames of
 * more than PT_ATROUS_NOALLOC_MAX_PIXELS pixels are refused with
 * PT_ERR_INVALID_ARG. The first call in each CUDA context looks up the
 * array's device address (make the first call on a device, and the first after
 * a cudaDeviceReset, before any stream capture). All calls share the
 * array: calls whose work overlaps on the GPU (other streams, other threads)
 * race and corrupt each other's output. Device buffers, enqueued on stream. */
#define PT_ATROUS_NOALLOC_MAX_PIXELS 262144
pt_status pt_denoise_atrous_device_noalloc(int width, int height, const float* d_color, const float* d_albedo,
                                           const float* d_normal, const float* d_variance, float* d_out,
                                           void* stream);

/* ---- measurement ------------------------------------------------------------------------
 * No counterpart in the reference: the L2 read rate the traversal roofline is
 * also reported against. Re-reads one device buffer of `bytes` (keep it
 * under the 126 MB L2) `reps` times per launch with 16-byte loads that bypass
 * L1; *gbs = bytes read per second over 10 launches, in GB/s. Allocates and
 * frees its own buffer; blocking. */
pt_status pt_measure_l2_read(size_t bytes, int reps, double* gbs);

/* ---- learned denoiser (no reference counterpart) ---------------------------------
 * A U-Net over 10 guide channels per pixel: radiance 3, albedo 3, normal 3 and
 * depth 1 (the renderer's 7-float aux gives albedo and normal,
 * pt_primary_depth_device the depth). Four levels of 32/64/96/128 channels, two
 * 3x3 convolutions + ReLU per level, 2x2 max pooling, nearest 2x upsampling
 * with skip concatenation, a final 3x3 convolution to log(1 + radiance).
 * bfloat16 activations, float accumulation, float master weights, Adam.
 *
 * Parameters: 15 convolutions in forward order (32->32, 32->32, 32->64,
 * 64->64, 64->96, 96->96, 96->128, 128->128, 224->96, 96->96, 160->64, 64->64,
 * 96->32, 32->32, 32->16), each weights [Cout][3][3][Cin] then bias [Cout], as
 * floats. The first layer's input channels 10..31 and the last layer's output
 * channels 3..15 are padding.
 *
 * Batched tensors (forward, training): NHWC float, input 10 channels, target
 * and output 3 (linear radiance); height and width multiples of 8. */
typedef struct pt_unet pt_unet;
pt_status pt_unet_create(uint64_t seed, pt_unet** out);
pt_status pt_unet_destroy(pt_unet* net);
size_t pt_unet_num_params(const pt_unet* net);
/* Copy the float parameters out / in (pt_unet_num_params floats). Both wait
 * for all work on the device first, so a training step in flight on any
 * stream finishes before the copy; blocking. */
pt_status pt_unet_get_params(const pt_unet* net, float* host_params);
pt_status pt_unet_set_params(pt_unet* net, const float* host_params);
/* 1 (default): convolutions with bfloat16 inputs run on the tensor cores where
 * the shape allows; 0: on the CUDA cores only. */
pt_status pt_unet_set_tensor_cores(pt_unet* net, int enable);
/* Waits for the network's work on stream; PT_ERR_TIMEOUT if a tensor-core
 * convolution gave up waiting for its operands since the last check. */
pt_status pt_unet_sync(pt_unet* net, void* stream);
pt_status pt_unet_forward(pt_unet* net, int batch, int height, int width, const float* d_input, float* d_output,
                          void* stream);
/* One Adam step (b1 0.9, b2 0.999, eps 1e-8) on the mean L1 distance between
 * log(1 + output) and log(1 + target); *loss (may be NULL) gets that loss
 * before the step. Synchronises stream. */
pt_status pt_unet_train_step(pt_unet* net, int batch, int height, int width, const float* d_input,
                             const float* d_target, float lr, float* loss, void* stream);
/* The loss and its gradients without a step (synchronous, default stream):
 * host_grads (NULL or pt_unet_num_params floats) in the parameter layout;
 * host_input_grad (NULL or batch*height*width*32 floats) with respect to the
 * network's padded input (log radiance, albedo, normal, log depth, zeros). */
pt_status pt_unet_loss_grads(pt_unet* net, int batch, int height, int width, const float* d_input,
                             const float* d_target, float* loss, float* host_grads, float* host_input_grad);
/* Denoises one frame (any size; padded internally to multiples of 8 by
 * repeating edge pixels): d_color 3 floats per pixel, d_aux the renderer's 7
 * floats per pixel, d_depth 1 float per pixel, all top row first; d_out 3
 * floats per pixel. Device buffers, enqueued on stream. */
pt_status pt_denoise_unet(pt_unet* net, int width, int height, const float* d_color, const float* d_aux,
                          const float* d_depth, float* d_out, void* stream);

/* ---- ground truth and images ------------------------------------------------------- */
/* Adds weight * d_frame[i] to d_sum[i] in FP64 (device buffers, enqueued on
 * stream): a progressive pass's per-pixel averages times its spp, for
 * ground-truth sums over many passes (no reference counterpart). */
pt_status pt_accumulate_pass(const float* d_frame, size_t n_floats, double weight, double* d_sum, void* stream);
/* write_image (include/image_write.hpp:15-33): PFM for a path ending in .pfm
 * (linear, bottom row first), else binary PPM of to_display bytes. linear is
 * 3 floats per pixel, top row first. */
pt_status pt_write_image(const char* path, int width, int height, const float* linear);
/* to_display (include/renderer.hpp:421-423): gamma 2, clamped, to a byte. */
uint8_t pt_to_display(float linear);

/* ---- batched rendering (no reference counterpart) ------------------------------ */
/* Many scenes of different size, resolution and spp rendered together: their
 * trees share one device arena and, with PT_BATCH_ONE_LAUNCH, one persistent
 * launch (captured in a CUDA graph) covers every scene's pixels. Each scene's
 * image is what pt_render would give for it (PT_RNG_SAMPLE streams). */
enum { PT_BATCH_AUTO = 0, PT_BATCH_ONE_LAUNCH = 1, PT_BATCH_PER_SCENE_MEGA = 2, PT_BATCH_PER_SCENE_WAVE = 3 };
typedef struct pt_batch_item {
    const pt_scene_desc* desc; /* with use_bvh set */
    pt_camera camera;
    int32_t width, height, spp, max_bounces;
    uint64_t seed;
} pt_batch_item;
typedef struct pt_batch_info {
    uint32_t n_scenes;
    int32_t strategy;   /* the one used (the autotuner's choice for PT_BATCH_AUTO) */
    int32_t threads;    /* block size of the single launch */
    int32_t tuned;
    uint64_t total_pixels, total_samples, device_bytes;
    double tune_ms[8];  /* autotuner timings: one launch at 64/128/256 threads per block, per-scene megakernel,
                           per-scene wavefront with 2^20, 2^19, 2^18 paths in flight, (unused) */
} pt_batch_info;
typedef struct pt_batch pt_batch;
/* Deep-copies the scenes into one arena. PT_BATCH_AUTO measures every
 * strategy on the first pt_batch_render and keeps the fastest (remembered
 * for batches of the same shape). */
pt_status pt_batch_create(const pt_batch_item* items, uint32_t n, int32_t strategy, pt_batch** out);
/* Renders every scene into the batch's device output, enqueued on stream
 * (NULL: the batch's own); rays_out (may be NULL) waits and returns the
 * ray count. */
pt_status pt_batch_render(pt_batch* batch, void* stream, uint64_t* rays_out);
/* Scene i's image in device memory (3 floats per pixel, top row first). */
pt_status pt_batch_output(const pt_batch* batch, uint32_t i, const float** d_image);
/* Copies scene i's image to host memory (waits for the batch). */
pt_status pt_batch_download(pt_batch* batch, uint32_t i, float* host);
/* Completion time of each scene in the last render, ms from its start. */
pt_status pt_batch_scene_times(pt_batch* batch, double* ms);
pt_status pt_batch_get_info(const pt_batch* batch, pt_batch_info* info);
pt_status pt_batch_destroy(pt_batch* batch);

/* ---- procedural scenes and ray sets (no reference counterpart) ---------------- */
/* Generators for the benchmark workloads and the reference's own scenes
 * (materials, field, room: include/renderer.hpp:158-208, 245-268). */
enum {
    PT_GEN_REF_MATERIALS = 0, /* make_scene(materials) */
    PT_GEN_REF_FIELD = 1,     /* make_scene(field) */
    PT_GEN_REF_ROOM = 3,      /* make_room_scene() */
    PT_GEN_RANDOM_SPHERES = 10, /* 22x22 random spheres + ground + light, seed */
    PT_GEN_ROOM_MESH = 11,      /* closed room + displaced icosphere (subdivisions = param) */
    PT_GEN_INSTANCES = 12,      /* 10,000 instances of three procedural meshes */
    PT_GEN_BATCH_SCENE = 13,    /* one scene of the 64-scene batch, by seed */
    PT_GEN_TEXTURED = 14,       /* the room with textured walls, sphere and instanced meshes, seed */
    PT_GEN_MESH_LIGHT = 15      /* the room lit by emissive triangle meshes, rough metal (extended NEE) */
};
typedef struct pt_gen_params {
    int32_t kind;
    int32_t param;      /* kind-specific: subdivisions, sphere count, instance count (0 = default) */
    uint64_t seed;
    int32_t use_bvh;    /* -1: the reference's default for the scene */
    int32_t width, height, spp; /* suggested render size (outputs; filled by pt_generate) */
} pt_gen_params;

typedef struct pt_generated pt_generated;
/* Builds a scene. params->width/height/spp are filled with the workload's
 * render size. */
pt_status pt_generate(pt_gen_params* params, pt_generated** out);
const pt_scene_desc* pt_generated_desc(const pt_generated* g);
const pt_camera* pt_generated_camera(const pt_generated* g);
void pt_generated_free(pt_generated* g);

/* n rays (6 floats each) with origins uniform in the box [lo, hi] and
 * directions uniform on the sphere, drawn from std::mt19937_64(seed) in a
 * fixed order (origin x, y, z, then z = 1 - 2u, phi = 2 pi v). */
pt_status pt_generate_rays(uint64_t seed, const float lo[3], const float hi[3], size_t n, float* rays);

#ifdef __cplusplus
}
#endif
#endif /* PHOTON_CUDA_H */
