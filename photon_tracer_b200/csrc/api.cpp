// The extern "C" entry points of libphoton_cuda (include/photon_cuda.h):
// scene upload, renders and ray queries, with every error turned into a
// pt_status and a message for pt_last_error(). No exception leaves this file.
#include <cuda_runtime.h>

#include <chrono>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "kernels.h"
#include "wavefront.h"
#include "scene_host.hpp"

namespace pt {

namespace {
thread_local std::string g_error;
}

void set_error(const std::string& msg) { g_error = msg; }
void clear_error() { g_error.clear(); }
pt_status fail(pt_status code, const std::string& msg) {
    g_error = msg;
    return code;
}
const char* error_text() { return g_error.c_str(); }

pt_status cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? PT_ERR_OUT_OF_MEMORY : PT_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace pt

using namespace pt;

// Device memory a scene keeps between host-buffer calls.
struct Scratch {
    void* ptr = nullptr;
    size_t bytes = 0;
    pt_status ensure(size_t want, const char* what) {
        if (want <= bytes) return PT_OK;
        release();
        if (cudaError_t e = cudaMalloc(&ptr, want)) {
            ptr = nullptr;
            return cuda_fail(e, what);
        }
        bytes = want;
        return PT_OK;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

struct pt_scene {
    PtSceneDev dev{};
    pt_scene_info info;
    int device = 0;
    int sms = 148;
    void* arena = nullptr;
    unsigned int* status = nullptr;    // device error word
    unsigned int* work = nullptr;      // megakernel work counter
    unsigned long long* rays = nullptr;
    cudaStream_t stream = nullptr;
    Scratch out, aux, states, in_rays, out_hits, counts, wave, sum;
    uint32_t* host_counts = nullptr;  // pinned, for the wavefront queue read-back
    int blocks_per_sm[6] = {0, 0, 0, 0, 0, 0};  // megakernel forms: aux, snapshot; extended light sampling
    uint32_t wave_slots = 0;                   // wavefront path-queue capacity; 0: kMaxWaveSlots
};

namespace {

pt_status check_device(int& device, int& sms) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(PT_ERR_NO_DEVICE, "no CUDA device");
    if (cudaGetDevice(&device) != cudaSuccess) return fail(PT_ERR_NO_DEVICE, "no current CUDA device");
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) return fail(PT_ERR_NO_DEVICE, "libphoton_cuda is built for sm_100a (B200) only");
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return PT_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

pt_status use_device(pt_scene* s) {
    if (cudaError_t e = cudaSetDevice(s->device)) return cuda_fail(e, "cudaSetDevice");
    return PT_OK;
}

// Waits for `stream`, then reads and clears the scene's device error word.
pt_status read_status(pt_scene* s, cudaStream_t stream) {
    if (cudaError_t e = cudaStreamSynchronize(stream)) return cuda_fail(e, "kernel");
    unsigned int st = 0;
    if (cudaError_t e = cudaMemcpy(&st, s->status, sizeof(st), cudaMemcpyDeviceToHost)) return cuda_fail(e, "status");
    if (st) {
        // Cleared on the scene's stream, so the clear is ordered before the
        // next kernel that may set a bit again.
        cudaMemsetAsync(s->status, 0, sizeof(unsigned int), stream);
        if (st & PT_DEV_ERR_STACK) return fail(PT_ERR_STACK_OVERFLOW, "a traversal stack overflowed on the device");
        if (st & PT_DEV_ERR_QUEUE) return fail(PT_ERR_QUEUE_OVERFLOW, "a wavefront queue overflowed on the device");
        if (st & PT_DEV_ERR_TIMEOUT) return fail(PT_ERR_TIMEOUT, "a device wait timed out");
    }
    return PT_OK;
}

pt_status check_settings(const pt_settings* st) {
    if (!st) return fail(PT_ERR_INVALID_ARG, "settings: null pointer");
    if (st->width < 2 || st->height < 2) return fail(PT_ERR_INVALID_ARG, "settings: width and height must be >= 2");
    if (int64_t(st->width) * st->height > (int64_t(1) << 30)) return fail(PT_ERR_INVALID_ARG, "settings: image too large");
    if (st->spp < 1) return fail(PT_ERR_INVALID_ARG, "settings: spp must be >= 1");
    if (st->max_bounces < 0) return fail(PT_ERR_INVALID_ARG, "settings: max_bounces must be >= 0");
    if (st->first_sample < 0) return fail(PT_ERR_INVALID_ARG, "settings: first_sample must be >= 0");
    if (st->rng != PT_RNG_SAMPLE && st->rng != PT_RNG_SNAPSHOT) return fail(PT_ERR_INVALID_ARG, "settings: unknown rng");
    if (st->rng == PT_RNG_SNAPSHOT && !st->rng_states)
        return fail(PT_ERR_INVALID_ARG, "settings: PT_RNG_SNAPSHOT needs rng_states");
    if (st->mode < PT_MODE_AUTO || st->mode > PT_MODE_WAVEFRONT)
        return fail(PT_ERR_INVALID_ARG, "settings: unknown mode");
    if (st->flags & ~int32_t(PT_FLAG_NEE_EXTENDED)) return fail(PT_ERR_INVALID_ARG, "settings: unknown flags");
    if ((st->flags & PT_FLAG_NEE_EXTENDED) && st->rng == PT_RNG_SNAPSHOT)
        return fail(PT_ERR_UNSUPPORTED, "settings: PT_FLAG_NEE_EXTENDED needs PT_RNG_SAMPLE streams");
    if ((st->flags & PT_FLAG_NEE_EXTENDED) && st->mode == PT_MODE_WAVEFRONT)
        return fail(PT_ERR_UNSUPPORTED, "settings: PT_FLAG_NEE_EXTENDED renders with the megakernel");
    return PT_OK;
}

PtRenderParams make_params(const pt_camera* cam, const pt_settings* st) {
    PtRenderParams p;
    std::memset(&p, 0, sizeof(p));
    std::memcpy(p.cam.origin, cam->origin, sizeof(p.cam.origin));
    std::memcpy(p.cam.llc, cam->lower_left, sizeof(p.cam.llc));
    std::memcpy(p.cam.horizontal, cam->horizontal, sizeof(p.cam.horizontal));
    std::memcpy(p.cam.vertical, cam->vertical, sizeof(p.cam.vertical));
    p.width = st->width;
    p.height = st->height;
    p.spp = st->spp;
    p.depth = st->max_bounces;
    p.seed = st->seed;
    p.first_sample = st->first_sample;
    p.rng_mode = st->rng;
    p.nee_ext = (st->flags & PT_FLAG_NEE_EXTENDED) ? 1 : 0;
    p.states = st->rng_states;
    p.row0 = 0;
    p.rows = st->height;
    p.flip = 1;
    return p;
}

// Paths the wavefront keeps in flight: one per pixel up to 2^20.
constexpr uint32_t kMaxWaveSlots = 1u << 20;

pt_status launch_render(pt_scene* s, PtRenderParams& p, int mode, cudaStream_t stream) {
    if (mode == PT_MODE_WAVEFRONT) {
        const uint64_t px = uint64_t(p.width) * uint64_t(p.rows);
        const uint32_t cap = s->wave_slots ? s->wave_slots : kMaxWaveSlots;
        const uint32_t slots = uint32_t(px < cap ? px : cap);
        if (pt_status e = s->wave.ensure(pt_wavefront_bytes(slots), "wavefront state")) return e;
        if (!s->host_counts)
            if (cudaError_t e = cudaMallocHost(&s->host_counts, 256)) return cuda_fail(e, "wavefront counters");
        if (cudaError_t e = pt_launch_wavefront(s->dev, p, s->wave.ptr, slots, s->sms, stream, s->host_counts))
            return cuda_fail(e, "wavefront");
        return PT_OK;
    }
    if (cudaError_t e = cudaMemsetAsync(s->work, 0, sizeof(unsigned int), stream)) return cuda_fail(e, "render");
    const int variant = p.nee_ext ? 4 + (p.aux ? 1 : 0) : (p.aux ? 1 : 0) + (p.rng_mode == PT_RNG_SNAPSHOT ? 2 : 0);
    PtLaunchShape shape;
    shape.threads = 128;
    if (!s->blocks_per_sm[variant])
        s->blocks_per_sm[variant] = pt_megakernel_blocks_per_sm(s->dev, shape.threads, p.aux != nullptr,
                                                                p.rng_mode == PT_RNG_SNAPSHOT, p.nee_ext != 0);
    shape.blocks = s->sms * s->blocks_per_sm[variant];
    p.work = s->work;
    if (cudaError_t e = pt_launch_megakernel(s->dev, p, shape, stream)) return cuda_fail(e, "megakernel launch");
    return PT_OK;
}

}  // namespace

void pt::set_wave_slots(pt_scene* s, uint32_t slots) { s->wave_slots = slots; }

namespace {

template <class T>
T* upload(char* base, size_t& off, const std::vector<T>& v, cudaError_t& err) {
    T* dst = reinterpret_cast<T*>(base + off);
    if (!v.empty() && err == cudaSuccess)
        err = cudaMemcpy(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    off += align256(v.size() * sizeof(T));
    return dst;
}

}  // namespace

extern "C" {

const char* pt_last_error(void) { return error_text(); }

const char* pt_version(void) { return "photon_cuda 0.1 (sm_100a)"; }

void pt_free(void* p) { std::free(p); }

pt_status pt_triangle_init(const float p0[3], const float p1[3], const float p2[3], const float* normals,
                           uint32_t material, pt_triangle* out) {
    clear_error();
    if (!p0 || !p1 || !p2 || !out) return fail(PT_ERR_INVALID_ARG, "pt_triangle_init: null pointer");
    *out = normals ? make_triangle(load(p0), load(p1), load(p2), load(normals), load(normals + 3), load(normals + 6),
                                   material)
                   : make_triangle(load(p0), load(p1), load(p2), material);
    return PT_OK;
}

pt_status pt_affine_inverse(const pt_affine* to_world, pt_affine* to_object) {
    clear_error();
    if (!to_world || !to_object) return fail(PT_ERR_INVALID_ARG, "pt_affine_inverse: null pointer");
    *to_object = affine_inverse(*to_world);
    return PT_OK;
}

pt_status pt_bvh_build(const float* boxes, uint32_t n, pt_bvh_node** nodes, uint32_t* n_nodes, uint32_t** order) {
    clear_error();
    if ((!boxes && n) || !nodes || !n_nodes || !order) return fail(PT_ERR_INVALID_ARG, "pt_bvh_build: null pointer");
    try {
        std::vector<pt_bvh_node> nv;
        std::vector<uint32_t> ov;
        build_bvh(boxes, n, nv, ov);
        *nodes = static_cast<pt_bvh_node*>(std::malloc(std::max<size_t>(1, nv.size()) * sizeof(pt_bvh_node)));
        *order = static_cast<uint32_t*>(std::malloc(std::max<size_t>(1, ov.size()) * sizeof(uint32_t)));
        if (!*nodes || !*order) {
            std::free(*nodes);
            std::free(*order);
            *nodes = nullptr;
            *order = nullptr;
            return fail(PT_ERR_OUT_OF_MEMORY, "pt_bvh_build: out of host memory");
        }
        if (!nv.empty()) std::memcpy(*nodes, nv.data(), nv.size() * sizeof(pt_bvh_node));
        if (!ov.empty()) std::memcpy(*order, ov.data(), ov.size() * sizeof(uint32_t));
        *n_nodes = uint32_t(nv.size());
        return PT_OK;
    } catch (const std::bad_alloc&) {
        return fail(PT_ERR_OUT_OF_MEMORY, "pt_bvh_build: out of host memory");
    }
}

pt_status pt_scene_create(const pt_scene_desc* desc, pt_scene** out) {
    clear_error();
    if (!desc || !out) return fail(PT_ERR_INVALID_ARG, "pt_scene_create: null pointer");
    *out = nullptr;
    // The description is checked and packed on the host first, so that its
    // errors are reported the same with or without a device.
    HostArena A;
    try {
        if (pt_status st = build_arena(*desc, A)) return st;
    } catch (const std::bad_alloc&) {
        return fail(PT_ERR_OUT_OF_MEMORY, "pt_scene_create: out of host memory");
    }
    int device = 0, sms = 0;
    if (pt_status st = check_device(device, sms)) return st;
    pt_scene* s = new (std::nothrow) pt_scene();
    if (!s) return fail(PT_ERR_OUT_OF_MEMORY, "pt_scene_create: out of host memory");
    s->device = device;
    s->sms = sms;
    const size_t bytes = align256(A.nodes.size() * 4) + align256(A.slots.size() * 4) + align256(A.islots.size() * 4) +
                         align256(A.large.size() * sizeof(float4)) + align256(A.large_mat.size() * 4) +
                         align256(A.sph.size() * sizeof(PtShadeSphere)) + align256(A.tri.size() * sizeof(PtShadeTri)) +
                         align256(A.inst.size() * sizeof(PtShadeInst)) + align256(A.mat.size() * sizeof(PtMaterial)) +
                         align256(A.lights.size() * sizeof(PtLight)) + align256(A.tri_uv.size() * 4) +
                         align256(A.tex.size() * sizeof(int4)) + align256(A.texels.size() * 4) +
                         align256(A.tri_lights.size() * sizeof(PtTriLight)) + align256(A.light_cdf.size() * 4) +
                         3 * 256;
    cudaError_t err = cudaMalloc(&s->arena, bytes);
    if (err != cudaSuccess) {
        delete s;
        return cuda_fail(err, "pt_scene_create: device allocation");
    }
    char* base = static_cast<char*>(s->arena);
    size_t off = 0;
    PtSceneDev& D = s->dev;
    std::memset(&D, 0, sizeof(D));
    D.nodes = reinterpret_cast<const float4*>(upload(base, off, A.nodes, err));
    D.slots = reinterpret_cast<const float4*>(upload(base, off, A.slots, err));
    D.islots = reinterpret_cast<const float4*>(upload(base, off, A.islots, err));
    D.large = upload(base, off, A.large, err);
    D.large_mat = upload(base, off, A.large_mat, err);
    D.sph = upload(base, off, A.sph, err);
    D.tri = upload(base, off, A.tri, err);
    D.inst = upload(base, off, A.inst, err);
    D.mat = upload(base, off, A.mat, err);
    D.lights = upload(base, off, A.lights, err);
    D.tri_lights = upload(base, off, A.tri_lights, err);
    D.light_cdf = upload(base, off, A.light_cdf, err);
    D.tri_uv = upload(base, off, A.tri_uv, err);
    D.tex = upload(base, off, A.tex, err);
    D.texels = upload(base, off, A.texels, err);
    D.has_textures = A.has_textures;
    D.ordered_boxes = ordered_boxes(A.nodes);
    D.stack_pack8 = stack_pack8(A.nodes);
    D.tree_kib = tree_kib(A.nodes, A.slots);
    s->status = reinterpret_cast<unsigned int*>(base + off);
    off += 256;
    s->work = reinterpret_cast<unsigned int*>(base + off);
    off += 256;
    s->rays = reinterpret_cast<unsigned long long*>(base + off);
    off += 256;
    if (err == cudaSuccess) err = cudaMemset(s->status, 0, 3 * 256);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        cudaFree(s->arena);
        delete s;
        return cuda_fail(err, "pt_scene_create: upload");
    }
    D.status = s->status;
    D.flat_root = A.flat_root;
    D.inst_root = A.inst_root;
    D.n_flat_slots = A.n_flat_slots;
    D.n_instances = A.n_instances;
    D.n_large = uint32_t(A.large.size());
    D.n_lights = uint32_t(A.lights.size());
    D.n_tri_lights = uint32_t(A.tri_lights.size());
    D.pick_uniform = A.pick_uniform;
    D.pick_power = A.pick_power;
    D.n_spheres = A.n_spheres;
    D.sky = A.sky;
    D.sample_lights = A.sample_lights;
    D.use_bvh = A.use_bvh;
    s->info.n_nodes = uint32_t(A.nodes.size() / 32);
    s->info.n_slots = uint32_t(A.slots.size() / 12);
    s->info.max_depth = A.max_depth;
    s->info.stack_entries = A.stack_entries;
    s->info.device_bytes = bytes;
    *out = s;
    return PT_OK;
}

pt_status pt_scene_destroy(pt_scene* s) {
    clear_error();
    if (!s) return PT_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    s->out.release();
    s->aux.release();
    s->sum.release();
    s->states.release();
    s->in_rays.release();
    s->out_hits.release();
    s->counts.release();
    s->wave.release();
    if (s->host_counts) cudaFreeHost(s->host_counts);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->arena) cudaFree(s->arena);
    delete s;
    return PT_OK;
}

pt_status pt_scene_get_info(const pt_scene* s, pt_scene_info* info) {
    clear_error();
    if (!s || !info) return fail(PT_ERR_INVALID_ARG, "pt_scene_get_info: null pointer");
    *info = s->info;
    return PT_OK;
}

pt_status pt_render_device(pt_scene* s, const pt_camera* cam, const pt_settings* st, float* d_out, float* d_aux,
                           uint64_t* d_rays, void* stream) {
    clear_error();
    if (!s || !cam || !d_out) return fail(PT_ERR_INVALID_ARG, "pt_render_device: null pointer");
    if (pt_status e = check_settings(st)) return e;
    if (pt_status e = use_device(s)) return e;
    PtRenderParams p = make_params(cam, st);
    p.out = d_out;
    p.aux = d_aux;
    p.rays = reinterpret_cast<unsigned long long*>(d_rays);
    return launch_render(s, p, st->mode, static_cast<cudaStream_t>(stream));
}

pt_status pt_sync(pt_scene* s, void* stream) {
    clear_error();
    if (!s) return fail(PT_ERR_INVALID_ARG, "pt_sync: null scene");
    if (pt_status e = use_device(s)) return e;
    return read_status(s, static_cast<cudaStream_t>(stream));
}

pt_status pt_render(pt_scene* s, const pt_camera* cam, const pt_settings* st, float* out, float* aux,
                    uint64_t* rays_out) {
    clear_error();
    if (!s || !cam || !out) return fail(PT_ERR_INVALID_ARG, "pt_render: null pointer");
    if (pt_status e = check_settings(st)) return e;
    if (pt_status e = use_device(s)) return e;
    const size_t px = size_t(st->width) * st->height;
    if (pt_status e = s->out.ensure(3 * px * sizeof(float), "pt_render: output")) return e;
    if (aux)
        if (pt_status e = s->aux.ensure(7 * px * sizeof(float), "pt_render: aux")) return e;
    PtRenderParams p = make_params(cam, st);
    cudaStream_t stream = s->stream;
    if (st->rng == PT_RNG_SNAPSHOT) {
        const size_t words = 4 * px * size_t(st->spp);
        if (pt_status e = s->states.ensure(words * 8, "pt_render: rng states")) return e;
        if (cudaError_t e = cudaMemcpyAsync(s->states.ptr, st->rng_states, words * 8, cudaMemcpyHostToDevice, stream))
            return cuda_fail(e, "pt_render: rng states");
        p.states = static_cast<const uint64_t*>(s->states.ptr);
    }
    p.out = static_cast<float*>(s->out.ptr);
    p.aux = aux ? static_cast<float*>(s->aux.ptr) : nullptr;
    p.rays = s->rays;
    if (cudaError_t e = cudaMemsetAsync(s->rays, 0, sizeof(unsigned long long), stream)) return cuda_fail(e, "pt_render");
    if (pt_status e = launch_render(s, p, st->mode, stream)) return e;
    if (cudaError_t e = cudaMemcpyAsync(out, p.out, 3 * px * sizeof(float), cudaMemcpyDeviceToHost, stream))
        return cuda_fail(e, "pt_render: output copy");
    if (aux)
        if (cudaError_t e = cudaMemcpyAsync(aux, p.aux, 7 * px * sizeof(float), cudaMemcpyDeviceToHost, stream))
            return cuda_fail(e, "pt_render: aux copy");
    unsigned long long rays = 0;
    if (cudaError_t e = cudaMemcpyAsync(&rays, s->rays, sizeof(rays), cudaMemcpyDeviceToHost, stream))
        return cuda_fail(e, "pt_render: ray count");
    if (pt_status e = read_status(s, stream)) return e;
    if (rays_out) *rays_out = rays;
    return PT_OK;
}

pt_status pt_render_progressive(pt_scene* s, const pt_camera* cam, const pt_settings* st, float* out,
                                pt_progress_fn progress, void* user, int32_t* samples_done, uint64_t* rays_out) {
    clear_error();
    if (!s || !cam || !out) return fail(PT_ERR_INVALID_ARG, "pt_render_progressive: null pointer");
    if (pt_status e = check_settings(st)) return e;
    if (st->rng != PT_RNG_SAMPLE) return fail(PT_ERR_INVALID_ARG, "pt_render_progressive: needs PT_RNG_SAMPLE");
    if (pt_status e = use_device(s)) return e;
    const size_t px = size_t(st->width) * st->height;
    if (pt_status e = s->out.ensure(3 * px * sizeof(float), "pt_render_progressive: frame")) return e;
    if (pt_status e = s->sum.ensure(3 * px * sizeof(double), "pt_render_progressive: sums")) return e;
    cudaStream_t stream = s->stream;
    float* frame = static_cast<float*>(s->out.ptr);
    double* sum = static_cast<double*>(s->sum.ptr);
    if (cudaError_t e = cudaMemsetAsync(sum, 0, 3 * px * sizeof(double), stream)) return cuda_fail(e, "render_progressive");
    if (cudaError_t e = cudaMemsetAsync(s->rays, 0, sizeof(unsigned long long), stream))
        return cuda_fail(e, "render_progressive");
    int done = 0, batch = 1;
    while (done < st->spp) {
        pt_settings step = *st;
        step.spp = std::min(batch, st->spp - done);
        step.first_sample = st->first_sample + done;
        PtRenderParams p = make_params(cam, &step);
        p.out = frame;
        p.rays = s->rays;
        const auto t0 = std::chrono::steady_clock::now();
        if (pt_status e = launch_render(s, p, step.mode, stream)) return e;
        if (pt_status e = pt_accumulate_pass(frame, 3 * px, double(step.spp), sum, stream)) return e;
        if (pt_status e = read_status(s, stream)) return e;  // waits for the step
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        done += step.spp;
        if (ms < 20 && batch < 64)
            batch *= 2;
        else if (ms > 60 && batch > 1)
            batch = std::max(1, batch >> 1);
        if (progress && done < st->spp && progress(user, done, st->spp) != 0) break;
    }
    if (cudaError_t e = pt_launch_mean_of_sum(sum, 3 * px, 1.0 / double(done), frame, stream))
        return cuda_fail(e, "render_progressive: mean");
    if (cudaError_t e = cudaMemcpyAsync(out, frame, 3 * px * sizeof(float), cudaMemcpyDeviceToHost, stream))
        return cuda_fail(e, "render_progressive: output copy");
    unsigned long long rays = 0;
    if (cudaError_t e = cudaMemcpyAsync(&rays, s->rays, sizeof(rays), cudaMemcpyDeviceToHost, stream))
        return cuda_fail(e, "render_progressive: ray count");
    if (pt_status e = read_status(s, stream)) return e;
    if (samples_done) *samples_done = done;
    if (rays_out) *rays_out = rays;
    return PT_OK;
}

pt_status pt_render_row(pt_scene* s, const pt_camera* cam, int j, int width, int height, int samples_per_pixel,
                        int max_bounces, float* out, uint64_t seed, int first_sample, float* aux) {
    clear_error();
    if (!s || !cam || !out) return fail(PT_ERR_INVALID_ARG, "pt_render_row: null pointer");
    if (j < 0 || j >= height) return fail(PT_ERR_INVALID_ARG, "pt_render_row: row out of range");
    pt_settings st;
    std::memset(&st, 0, sizeof(st));
    st.width = width;
    st.height = height;
    st.spp = samples_per_pixel;
    st.max_bounces = max_bounces;
    st.seed = seed;
    st.first_sample = first_sample;
    if (pt_status e = check_settings(&st)) return e;
    if (pt_status e = use_device(s)) return e;
    if (pt_status e = s->out.ensure(3 * size_t(width) * sizeof(float), "pt_render_row: output")) return e;
    if (aux)
        if (pt_status e = s->aux.ensure(7 * size_t(width) * sizeof(float), "pt_render_row: aux")) return e;
    PtRenderParams p = make_params(cam, &st);
    p.row0 = j;
    p.rows = 1;
    p.flip = 0;
    p.out = static_cast<float*>(s->out.ptr);
    p.aux = aux ? static_cast<float*>(s->aux.ptr) : nullptr;
    cudaStream_t stream = s->stream;
    if (pt_status e = launch_render(s, p, PT_MODE_MEGAKERNEL, stream)) return e;
    if (cudaError_t e = cudaMemcpyAsync(out, p.out, 3 * size_t(width) * sizeof(float), cudaMemcpyDeviceToHost, stream))
        return cuda_fail(e, "pt_render_row: output copy");
    if (aux)
        if (cudaError_t e = cudaMemcpyAsync(aux, p.aux, 7 * size_t(width) * sizeof(float), cudaMemcpyDeviceToHost, stream))
            return cuda_fail(e, "pt_render_row: aux copy");
    return read_status(s, stream);
}

pt_status pt_trace_closest_device(pt_scene* s, const float* d_rays, size_t n, float tmin, float tmax, pt_hit* d_hits,
                                  void* stream) {
    clear_error();
    if (!s || (n && (!d_rays || !d_hits))) return fail(PT_ERR_INVALID_ARG, "pt_trace_closest_device: null pointer");
    if (pt_status e = use_device(s)) return e;
    if (cudaError_t e = pt_launch_trace_closest(s->dev, d_rays, n, tmin, tmax, d_hits, static_cast<cudaStream_t>(stream)))
        return cuda_fail(e, "trace_closest launch");
    return PT_OK;
}

pt_status pt_trace_any_device(pt_scene* s, const float* d_rays, size_t n, float tmin, float tmax, uint8_t* d_occ,
                              void* stream) {
    clear_error();
    if (!s || (n && (!d_rays || !d_occ))) return fail(PT_ERR_INVALID_ARG, "pt_trace_any_device: null pointer");
    if (pt_status e = use_device(s)) return e;
    if (cudaError_t e = pt_launch_trace_any(s->dev, d_rays, n, tmin, tmax, d_occ, static_cast<cudaStream_t>(stream)))
        return cuda_fail(e, "trace_any launch");
    return PT_OK;
}

pt_status pt_primary_depth_device(pt_scene* s, const pt_camera* cam, int width, int height, float* d_depth,
                                  void* stream) {
    clear_error();
    if (!s || !cam || !d_depth) return fail(PT_ERR_INVALID_ARG, "pt_primary_depth_device: null pointer");
    if (width < 2 || height < 2) return fail(PT_ERR_INVALID_ARG, "pt_primary_depth_device: width and height must be >= 2");
    if (pt_status e = use_device(s)) return e;
    pt_settings st{};
    st.width = width;
    st.height = height;
    const PtRenderParams p = make_params(cam, &st);
    if (cudaError_t e = pt_launch_primary_depth(s->dev, p.cam, width, height, d_depth, static_cast<cudaStream_t>(stream)))
        return cuda_fail(e, "primary_depth launch");
    return PT_OK;
}

pt_status pt_trace_closest(pt_scene* s, const float* rays, size_t n, float tmin, float tmax, pt_hit* hits) {
    clear_error();
    if (!s || (n && (!rays || !hits))) return fail(PT_ERR_INVALID_ARG, "pt_trace_closest: null pointer");
    if (pt_status e = use_device(s)) return e;
    if (n == 0) return PT_OK;
    cudaStream_t stream = s->stream;
    if (pt_status e = s->in_rays.ensure(n * 24, "pt_trace_closest: rays")) return e;
    if (pt_status e = s->out_hits.ensure(n * sizeof(pt_hit), "pt_trace_closest: hits")) return e;
    if (cudaError_t e = cudaMemcpyAsync(s->in_rays.ptr, rays, n * 24, cudaMemcpyHostToDevice, stream))
        return cuda_fail(e, "pt_trace_closest: copy");
    if (cudaError_t e = pt_launch_trace_closest(s->dev, static_cast<const float*>(s->in_rays.ptr), n, tmin, tmax,
                                                s->out_hits.ptr, stream))
        return cuda_fail(e, "trace_closest launch");
    if (cudaError_t e = cudaMemcpyAsync(hits, s->out_hits.ptr, n * sizeof(pt_hit), cudaMemcpyDeviceToHost, stream))
        return cuda_fail(e, "pt_trace_closest: copy back");
    return read_status(s, stream);
}

pt_status pt_trace_any(pt_scene* s, const float* rays, size_t n, float tmin, float tmax, uint8_t* occ) {
    clear_error();
    if (!s || (n && (!rays || !occ))) return fail(PT_ERR_INVALID_ARG, "pt_trace_any: null pointer");
    if (pt_status e = use_device(s)) return e;
    if (n == 0) return PT_OK;
    cudaStream_t stream = s->stream;
    if (pt_status e = s->in_rays.ensure(n * 24, "pt_trace_any: rays")) return e;
    if (pt_status e = s->out_hits.ensure(n, "pt_trace_any: result")) return e;
    if (cudaError_t e = cudaMemcpyAsync(s->in_rays.ptr, rays, n * 24, cudaMemcpyHostToDevice, stream))
        return cuda_fail(e, "pt_trace_any: copy");
    if (cudaError_t e = pt_launch_trace_any(s->dev, static_cast<const float*>(s->in_rays.ptr), n, tmin, tmax,
                                            static_cast<uint8_t*>(s->out_hits.ptr), stream))
        return cuda_fail(e, "trace_any launch");
    if (cudaError_t e = cudaMemcpyAsync(occ, s->out_hits.ptr, n, cudaMemcpyDeviceToHost, stream))
        return cuda_fail(e, "pt_trace_any: copy back");
    return read_status(s, stream);
}

pt_status pt_trace_count(pt_scene* s, const float* rays, size_t n, float tmin, float tmax, uint64_t counts[5]) {
    clear_error();
    if (!s || !counts || (n && !rays)) return fail(PT_ERR_INVALID_ARG, "pt_trace_count: null pointer");
    if (pt_status e = use_device(s)) return e;
    cudaStream_t stream = s->stream;
    if (pt_status e = s->in_rays.ensure(std::max<size_t>(1, n) * 24, "pt_trace_count: rays")) return e;
    if (pt_status e = s->counts.ensure(5 * sizeof(unsigned long long), "pt_trace_count: counts")) return e;
    if (cudaError_t e = cudaMemsetAsync(s->counts.ptr, 0, 5 * sizeof(unsigned long long), stream))
        return cuda_fail(e, "pt_trace_count");
    if (n) {
        if (cudaError_t e = cudaMemcpyAsync(s->in_rays.ptr, rays, n * 24, cudaMemcpyHostToDevice, stream))
            return cuda_fail(e, "pt_trace_count: copy");
        if (cudaError_t e = pt_launch_trace_count(s->dev, static_cast<const float*>(s->in_rays.ptr), n, tmin, tmax,
                                                  static_cast<unsigned long long*>(s->counts.ptr), stream))
            return cuda_fail(e, "trace_count launch");
    }
    unsigned long long c[5];
    if (cudaError_t e = cudaMemcpyAsync(c, s->counts.ptr, sizeof(c), cudaMemcpyDeviceToHost, stream))
        return cuda_fail(e, "pt_trace_count: copy back");
    if (pt_status e = read_status(s, stream)) return e;
    for (int k = 0; k < 5; ++k) counts[k] = c[k];
    return PT_OK;
}

}  // extern "C"
