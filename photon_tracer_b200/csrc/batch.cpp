// Host side of the batched renderer: merges many scenes into one arena,
// launches them together (or one by one), and picks how by measuring.
//
// Merging: each scene is repacked as for pt_scene_create, then appended to
// the shared arrays with every index rebased -- child nodes, leaf slots,
// instance slots, mesh roots, shading records, materials -- so the kernels
// see one arena and a scene is only its roots, its ranges of large spheres
// and lights, and its frame (batch.h).
//
// Strategies (pt_batch_create's `strategy`, or chosen by the autotuner):
//   PT_BATCH_ONE_LAUNCH      one persistent launch over every scene's pixels,
//                            captured once in a CUDA graph and replayed;
//   PT_BATCH_PER_SCENE_MEGA  one megakernel launch per scene (also a graph);
//   PT_BATCH_PER_SCENE_WAVE  the wavefront renderer, scene after scene.
// The autotuner times every strategy (and 64/128/256-thread blocks for the
// single launch) on the batch itself the first time it is rendered, keeps
// the fastest, and remembers the choice for batches with the same shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "batch.h"
#include "scene_host.hpp"

namespace pt {
pt_status cuda_fail(cudaError_t e, const char* what);
}
using namespace pt;

struct pt_batch {
    int device = 0, sms = 148;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    PtSceneDev dev{};
    std::vector<PtBatchScene> scenes;
    std::vector<pt_batch_item> items;
    PtBatchScene* d_scenes = nullptr;
    PtSceneDev* d_views = nullptr;  // per scene: the arena as that scene alone
    float* d_out = nullptr;
    size_t out_floats = 0;
    unsigned int* d_work = nullptr;
    unsigned int* d_done = nullptr;
    unsigned long long* d_done_ns = nullptr;
    unsigned long long* d_start = nullptr;
    unsigned long long* d_rays = nullptr;
    unsigned int* d_status = nullptr;
    uint32_t total_items = 0;
    uint64_t total_pixels = 0, total_samples = 0, total_tris = 0;
    std::vector<pt_scene*> singles;  // per-scene scenes for the per-scene strategies
    cudaStream_t stream = nullptr;
    cudaGraphExec_t one_graph[3] = {nullptr, nullptr, nullptr};  // the single launch at 64, 128, 256 threads
    int strategy = PT_BATCH_AUTO, threads = 128;
    uint32_t wave_slots = 0;  // per-scene wavefront: paths in flight (0: the library's default, 2^20)
    bool tuned = false;
    double tune_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    std::vector<cudaEvent_t> scene_events;  // per-scene completion (per-scene strategies)
    cudaEvent_t start_event = nullptr;
    cudaEvent_t done_event = nullptr;  // recorded on the render's stream after its last launch
    int last_strategy = 0;
};

namespace {

std::mutex g_tune_lock;
struct TuneChoice {
    int strategy, threads;
    uint32_t wave_slots;
};
std::map<std::string, TuneChoice> g_tune_cache;  // batch shape -> the autotuner's choice

float ubits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
uint32_t bitsf(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Appends src to dst with every index rebased; returns the scene's roots and ranges.
PtBatchScene merge(HostArena& dst, const HostArena& src) {
    const uint32_t node_base = uint32_t(dst.nodes.size() / 32), slot_base = uint32_t(dst.slots.size() / 12),
                   islot_base = uint32_t(dst.islots.size() / 16), sph_base = uint32_t(dst.sph.size()),
                   tri_base = uint32_t(dst.tri.size()), inst_base = uint32_t(dst.inst.size()),
                   mat_base = uint32_t(dst.mat.size()), large_base = uint32_t(dst.large.size()),
                   light_base = uint32_t(dst.lights.size()), tex_base = uint32_t(dst.tex.size()),
                   texel_base = uint32_t(dst.texels.size());
    const float inf = std::numeric_limits<float>::infinity();
    for (size_t n = 0; n < src.nodes.size(); n += 32) {
        float rec[32];
        std::copy(src.nodes.begin() + n, src.nodes.begin() + n + 32, rec);
        for (int c = 0; c < 4; ++c) {
            const uint32_t count = bitsf(rec[28 + c]);
            uint32_t first = bitsf(rec[24 + c]);
            if (count & PT_COUNT_MASK) first += (count & PT_LEAF_INSTANCES) ? islot_base : slot_base;
            else if (rec[c] != inf) first += node_base;
            rec[24 + c] = ubits(first);
        }
        dst.nodes.insert(dst.nodes.end(), rec, rec + 32);
    }
    for (size_t k = 0; k < src.slots.size() / 12; ++k) {
        float s[12];
        std::copy(src.slots.begin() + 12 * k, src.slots.begin() + 12 * k + 12, s);
        if (k < src.n_flat_slots) {  // flat primitives: original numbers index the shading arrays
            const uint32_t ref = bitsf(s[9]);
            s[9] = ubits((ref & PT_SLOT_SPHERE) ? (((ref & ~PT_SLOT_SPHERE) + sph_base) | PT_SLOT_SPHERE)
                                                : ref + tri_base);
        }
        dst.slots.insert(dst.slots.end(), s, s + 12);
    }
    for (size_t k = 0; k < src.islots.size() / 16; ++k) {
        float s[16];
        std::copy(src.islots.begin() + 16 * k, src.islots.begin() + 16 * k + 16, s);
        s[12] = ubits(bitsf(s[12]) + node_base);
        s[13] = ubits(bitsf(s[13]) + inst_base);
        dst.islots.insert(dst.islots.end(), s, s + 16);
    }
    for (size_t i = 0; i < src.large.size(); ++i) {
        dst.large.push_back(src.large[i]);
        dst.large_mat.push_back(src.large_mat[i] + mat_base);
    }
    for (PtShadeSphere s : src.sph) {
        s.mat += mat_base;
        dst.sph.push_back(s);
    }
    for (PtShadeTri t : src.tri) {
        t.n0_mat.w = ubits(bitsf(t.n0_mat.w) + mat_base);
        dst.tri.push_back(t);
    }
    for (PtShadeInst in : src.inst) {
        in.tri_base += tri_base;
        if (in.material != PT_NONE) in.material += mat_base;
        dst.inst.push_back(in);
    }
    for (PtMaterial m : src.mat) {
        const uint32_t t = bitsf(m.ior_flags.z);
        if (t != PT_NONE) m.ior_flags.z = ubits(t + tex_base);
        dst.mat.push_back(m);
    }
    dst.lights.insert(dst.lights.end(), src.lights.begin(), src.lights.end());
    dst.tri_uv.insert(dst.tri_uv.end(), src.tri_uv.begin(), src.tri_uv.end());
    for (int4 t : src.tex) {
        t.z += int(texel_base);
        dst.tex.push_back(t);
    }
    dst.texels.insert(dst.texels.end(), src.texels.begin(), src.texels.end());
    dst.has_textures |= src.has_textures;
    PtBatchScene b;
    std::memset(&b, 0, sizeof(b));
    b.flat_root = src.flat_root == PT_NONE ? PT_NONE : src.flat_root + node_base;
    b.inst_root = src.inst_root == PT_NONE ? PT_NONE : src.inst_root + node_base;
    b.large_base = large_base;
    b.n_large = uint32_t(src.large.size());
    b.light_base = light_base;
    b.n_lights = uint32_t(src.lights.size());
    b.sky = uint32_t(src.sky);
    b.sample_lights = uint32_t(src.sample_lights);
    return b;
}

template <class T>
T* upload(char* base, size_t& off, const std::vector<T>& v, cudaError_t& err) {
    T* dst = reinterpret_cast<T*>(base + off);
    if (!v.empty() && err == cudaSuccess) err = cudaMemcpy(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    off += align256(v.size() * sizeof(T));
    return dst;
}

pt_status enqueue_one_launch(pt_batch* b, int threads, cudaStream_t stream) {
    PtBatchLaunch L;
    L.scenes = b->d_scenes;
    L.views = b->d_views;
    L.n_scenes = uint32_t(b->scenes.size());
    L.total_items = b->total_items;
    L.out = b->d_out;
    L.work = b->d_work;
    L.done_pixels = b->d_done;
    L.done_ns = b->d_done_ns;
    L.start_ns = b->d_start;
    L.rays = b->d_rays;
    L.any_instances = 0;
    for (const PtBatchScene& sc : b->scenes) L.any_instances |= sc.inst_root != PT_NONE ? 1 : 0;
    cudaError_t e = cudaMemsetAsync(b->d_work, 0, sizeof(unsigned int), stream);
    if (!e) e = cudaMemsetAsync(b->d_done, 0, b->scenes.size() * sizeof(unsigned int), stream);
    if (!e) e = cudaMemsetAsync(b->d_start, 0xff, sizeof(unsigned long long), stream);
    if (!e) e = pt_launch_batch(b->dev, L, threads, b->sms, stream);
    return e ? cuda_fail(e, "batch launch") : PT_OK;
}

pt_status enqueue_per_scene(pt_batch* b, int mode, cudaStream_t stream, bool record) {
    if (record && b->start_event) cudaEventRecord(b->start_event, stream);
    for (size_t i = 0; i < b->items.size(); ++i) {
        const pt_batch_item& it = b->items[i];
        pt_settings st;
        std::memset(&st, 0, sizeof(st));
        st.width = it.width;
        st.height = it.height;
        st.spp = it.spp;
        st.max_bounces = it.max_bounces;
        st.seed = it.seed;
        st.mode = mode;
        st.rng = PT_RNG_SAMPLE;
        if (pt_status s = pt_render_device(b->singles[i], &it.camera, &st, b->d_out + b->scenes[i].out_offset, nullptr,
                                           reinterpret_cast<uint64_t*>(b->d_rays), stream))
            return s;
        if (record && i < b->scene_events.size()) cudaEventRecord(b->scene_events[i], stream);
    }
    return PT_OK;
}

// Captures `body` on the batch's stream into an executable graph.
template <class Body>
pt_status capture(pt_batch* b, cudaGraphExec_t* exec, Body&& body) {
    cudaGraph_t g = nullptr;
    if (cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal))
        return cuda_fail(e, "graph capture");
    const pt_status st = body(b->stream);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e) return cuda_fail(e, "graph capture");
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    return e ? cuda_fail(e, "graph instantiate") : PT_OK;
}

pt_status run_strategy(pt_batch* b, int strategy, int threads, cudaStream_t stream) {
    b->last_strategy = strategy;
    if (strategy == PT_BATCH_ONE_LAUNCH) {
        const int slot = threads == 64 ? 0 : threads == 256 ? 2 : 1;
        if (!b->one_graph[slot])
            if (pt_status s = capture(b, &b->one_graph[slot],
                                      [&](cudaStream_t cs) { return enqueue_one_launch(b, threads, cs); }))
                return s;
        if (cudaError_t e = cudaGraphLaunch(b->one_graph[slot], stream)) return cuda_fail(e, "batch graph launch");
        return PT_OK;
    }
    if (strategy == PT_BATCH_PER_SCENE_MEGA) return enqueue_per_scene(b, PT_MODE_MEGAKERNEL, stream, true);
    for (pt_scene* s : b->singles) set_wave_slots(s, b->wave_slots);
    return enqueue_per_scene(b, PT_MODE_WAVEFRONT, stream, true);
}

double time_ms(pt_batch* b, int strategy, int threads) {
    cudaEvent_t a, z;
    cudaEventCreate(&a);
    cudaEventCreate(&z);
    cudaEventRecord(a, b->stream);
    const pt_status st = run_strategy(b, strategy, threads, b->stream);
    cudaEventRecord(z, b->stream);
    cudaEventSynchronize(z);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, z);
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    return st ? -double(st) : double(ms);
}

std::string shape_key(const pt_batch* b) {
    return std::to_string(b->scenes.size()) + ":" + std::to_string(b->total_pixels) + ":" +
           std::to_string(b->total_samples) + ":" + std::to_string(b->total_tris);
}

pt_status tune(pt_batch* b) {
    {
        std::lock_guard<std::mutex> lock(g_tune_lock);
        auto it = g_tune_cache.find(shape_key(b));
        if (it != g_tune_cache.end()) {
            b->strategy = it->second.strategy;
            b->threads = it->second.threads;
            b->wave_slots = it->second.wave_slots;
            b->tuned = true;
            return PT_OK;
        }
    }
    // Every candidate once to warm up, then timed: the single launch at three
    // block shapes, per-scene megakernel launches, and per-scene wavefronts
    // at three path-queue capacities.
    struct Cand {
        int strategy, threads;
        uint32_t wave_slots;
        int slot;
    };
    const Cand cands[7] = {{PT_BATCH_ONE_LAUNCH, 64, 0, 0},          {PT_BATCH_ONE_LAUNCH, 128, 0, 1},
                           {PT_BATCH_ONE_LAUNCH, 256, 0, 2},         {PT_BATCH_PER_SCENE_MEGA, 128, 0, 3},
                           {PT_BATCH_PER_SCENE_WAVE, 128, 1u << 20, 4}, {PT_BATCH_PER_SCENE_WAVE, 128, 1u << 19, 5},
                           {PT_BATCH_PER_SCENE_WAVE, 128, 1u << 18, 6}};
    const uint32_t keep_slots = b->wave_slots;
    uint32_t best_slots = keep_slots;
    double best = 1e30;
    pt_status first_error = PT_OK;
    std::string first_message;
    bool any = false;
    for (const Cand& c : cands) {
        b->wave_slots = c.wave_slots;
        double ms = time_ms(b, c.strategy, c.threads);
        if (ms >= 0) ms = time_ms(b, c.strategy, c.threads);
        if (ms < 0) {  // the candidate failed: keep the first failure's status and message
            if (first_error == PT_OK) {
                first_error = static_cast<pt_status>(int(-ms));
                first_message = pt_last_error();
            }
            b->tune_ms[c.slot] = 1e30;
            continue;
        }
        any = true;
        b->tune_ms[c.slot] = ms;
        if (ms < best) {
            best = ms;
            b->strategy = c.strategy;
            b->threads = c.threads;
            best_slots = c.wave_slots;
        }
    }
    b->wave_slots = any ? best_slots : keep_slots;
    if (!any) return fail(first_error, first_message.c_str());
    b->tuned = true;
    std::lock_guard<std::mutex> lock(g_tune_lock);
    g_tune_cache[shape_key(b)] = {b->strategy, b->threads, b->wave_slots};
    return PT_OK;
}

}  // namespace

extern "C" {

pt_status pt_batch_create(const pt_batch_item* items, uint32_t n, int32_t strategy, pt_batch** out) {
    clear_error();
    if (!items || !out || n == 0) return fail(PT_ERR_INVALID_ARG, "pt_batch_create: null pointer or empty batch");
    if (strategy < PT_BATCH_AUTO || strategy > PT_BATCH_PER_SCENE_WAVE)
        return fail(PT_ERR_INVALID_ARG, "pt_batch_create: unknown strategy");
    *out = nullptr;
    int device = 0, sms = 148, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PT_ERR_NO_DEVICE, "no CUDA device");
    cudaGetDevice(&device);
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) return fail(PT_ERR_NO_DEVICE, "libphoton_cuda is built for sm_100a (B200) only");
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);

    pt_batch* b = new (std::nothrow) pt_batch();
    if (!b) return fail(PT_ERR_OUT_OF_MEMORY, "pt_batch_create: out of host memory");
    std::unique_ptr<pt_batch, void (*)(pt_batch*)> guard(b, [](pt_batch* p) { pt_batch_destroy(p); });
    b->device = device;
    b->sms = sms;
    b->strategy = strategy;
    HostArena all;
    uint64_t out_floats = 0;
    uint32_t items_total = 0;
    uint32_t stack_need = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const pt_batch_item& it = items[i];
        if (!it.desc) return fail(PT_ERR_INVALID_ARG, "pt_batch_create: item without a scene");
        if (it.width < 2 || it.height < 2 || it.spp < 1 || it.max_bounces < 0)
            return fail(PT_ERR_INVALID_ARG, "pt_batch_create: bad frame size, spp or depth");
        if (!it.desc->use_bvh) return fail(PT_ERR_UNSUPPORTED, "pt_batch_create: batched scenes need their BVH");
        HostArena A;
        try {
            if (pt_status st = build_arena(*it.desc, A)) return st;
        } catch (const std::bad_alloc&) {
            return fail(PT_ERR_OUT_OF_MEMORY, "pt_batch_create: out of host memory");
        }
        stack_need = std::max(stack_need, A.stack_entries);
        PtBatchScene s = merge(all, A);
        const uint32_t tiles_x = uint32_t((it.width + 7) / 8), tiles_y = uint32_t((it.height + 3) / 4);
        s.width = uint32_t(it.width);
        s.height = uint32_t(it.height);
        s.spp = uint32_t(it.spp);
        s.depth = uint32_t(it.max_bounces);
        s.seed = it.seed;
        s.out_offset = out_floats;
        s.tiles_x = tiles_x;
        s.item_base = items_total;
        std::memcpy(s.cam, it.camera.origin, 12);
        std::memcpy(s.cam + 3, it.camera.lower_left, 12);
        std::memcpy(s.cam + 6, it.camera.horizontal, 12);
        std::memcpy(s.cam + 9, it.camera.vertical, 12);
        if (uint64_t(items_total) + uint64_t(tiles_x) * tiles_y * 32 >= (uint64_t(1) << 31))
            return fail(PT_ERR_INVALID_ARG, "pt_batch_create: too many pixels in one batch");
        items_total += tiles_x * tiles_y * 32;
        out_floats += 3 * uint64_t(it.width) * uint64_t(it.height);
        b->scenes.push_back(s);
        b->items.push_back(it);
        b->total_pixels += uint64_t(it.width) * it.height;
        b->total_samples += uint64_t(it.width) * it.height * uint64_t(it.spp);
        b->total_tris += it.desc->n_triangles;
    }
    b->total_items = items_total;
    b->out_floats = out_floats;
    all.n_flat_slots = 0;
    const size_t bytes = align256(all.nodes.size() * 4) + align256(all.slots.size() * 4) + align256(all.islots.size() * 4) +
                         align256(all.large.size() * sizeof(float4)) + align256(all.large_mat.size() * 4) +
                         align256(all.sph.size() * sizeof(PtShadeSphere)) + align256(all.tri.size() * sizeof(PtShadeTri)) +
                         align256(all.inst.size() * sizeof(PtShadeInst)) + align256(all.mat.size() * sizeof(PtMaterial)) +
                         align256(all.lights.size() * sizeof(PtLight)) + align256(all.tri_uv.size() * 4) +
                         align256(all.tex.size() * sizeof(int4)) + align256(all.texels.size() * 4) +
                         align256(n * sizeof(PtBatchScene)) + align256(n * sizeof(PtSceneDev)) +
                         align256(out_floats * 4) + align256(n * 4) + align256(n * 8) + 4 * 256;
    cudaError_t err = cudaMalloc(&b->arena, bytes);
    if (err) return cuda_fail(err, "pt_batch_create: device allocation");
    b->arena_bytes = bytes;
    char* base = static_cast<char*>(b->arena);
    size_t off = 0;
    PtSceneDev& D = b->dev;
    std::memset(&D, 0, sizeof(D));
    D.nodes = reinterpret_cast<const float4*>(upload(base, off, all.nodes, err));
    D.slots = reinterpret_cast<const float4*>(upload(base, off, all.slots, err));
    D.islots = reinterpret_cast<const float4*>(upload(base, off, all.islots, err));
    D.large = upload(base, off, all.large, err);
    D.large_mat = upload(base, off, all.large_mat, err);
    D.sph = upload(base, off, all.sph, err);
    D.tri = upload(base, off, all.tri, err);
    D.inst = upload(base, off, all.inst, err);
    D.mat = upload(base, off, all.mat, err);
    D.lights = upload(base, off, all.lights, err);
    D.tri_uv = upload(base, off, all.tri_uv, err);
    D.tex = upload(base, off, all.tex, err);
    D.texels = upload(base, off, all.texels, err);
    D.has_textures = all.has_textures;
    D.ordered_boxes = ordered_boxes(all.nodes);
    D.stack_pack8 = stack_pack8(all.nodes);
    D.tree_kib = tree_kib(all.nodes, all.slots);
    b->d_scenes = upload(base, off, b->scenes, err);
    b->d_views = reinterpret_cast<PtSceneDev*>(base + off);
    off += align256(n * sizeof(PtSceneDev));
    b->d_out = reinterpret_cast<float*>(base + off);
    off += align256(out_floats * 4);
    b->d_done = reinterpret_cast<unsigned int*>(base + off);
    off += align256(n * 4);
    b->d_done_ns = reinterpret_cast<unsigned long long*>(base + off);
    off += align256(n * 8);
    b->d_work = reinterpret_cast<unsigned int*>(base + off);
    b->d_start = reinterpret_cast<unsigned long long*>(base + off + 256);
    b->d_rays = reinterpret_cast<unsigned long long*>(base + off + 512);
    b->d_status = reinterpret_cast<unsigned int*>(base + off + 768);
    if (!err) err = cudaMemset(base + off, 0, 4 * 256);
    if (!err) err = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (!err) err = cudaEventCreate(&b->start_event);
    if (!err) err = cudaEventCreateWithFlags(&b->done_event, cudaEventDisableTiming);
    for (uint32_t i = 0; i < n && !err; ++i) {
        cudaEvent_t ev;
        err = cudaEventCreate(&ev);
        if (!err) b->scene_events.push_back(ev);
    }
    if (err) return cuda_fail(err, "pt_batch_create: upload");
    D.status = b->d_status;
    D.use_bvh = 1;
    D.flat_root = D.inst_root = PT_NONE;
    {
        // each scene's view of the merged arena: its roots, its ranges of
        // large spheres and lights, its flags
        std::vector<PtSceneDev> views(n, D);
        for (uint32_t i = 0; i < n; ++i) {
            const PtBatchScene& sc = b->scenes[i];
            PtSceneDev& v = views[i];
            v.flat_root = sc.flat_root;
            v.inst_root = sc.inst_root;
            v.large = D.large + sc.large_base;
            v.large_mat = D.large_mat + sc.large_base;
            v.n_large = sc.n_large;
            v.lights = D.lights + sc.light_base;
            v.n_lights = sc.n_lights;
            v.sky = int(sc.sky);
            v.sample_lights = int(sc.sample_lights);
        }
        err = cudaMemcpy(b->d_views, views.data(), n * sizeof(PtSceneDev), cudaMemcpyHostToDevice);
        if (err) return cuda_fail(err, "pt_batch_create: scene views");
    }
    if (stack_need > PT_STACK_MAX) return fail(PT_ERR_STACK_OVERFLOW, "pt_batch_create: a scene's BVH is too deep");
    // Per-scene scenes for the strategies that launch scene by scene.
    if (strategy != PT_BATCH_ONE_LAUNCH) {
        for (uint32_t i = 0; i < n; ++i) {
            pt_scene* s = nullptr;
            if (pt_status st = pt_scene_create(items[i].desc, &s)) return st;
            b->singles.push_back(s);
        }
    }
    *out = guard.release();
    return PT_OK;
}

pt_status pt_batch_render(pt_batch* b, void* stream_, uint64_t* rays_out) {
    clear_error();
    if (!b) return fail(PT_ERR_INVALID_ARG, "pt_batch_render: null batch");
    if (cudaError_t e = cudaSetDevice(b->device)) return cuda_fail(e, "cudaSetDevice");
    if (b->strategy == PT_BATCH_AUTO && !b->tuned)
        if (pt_status st = tune(b)) return st;
    cudaStream_t stream = stream_ ? static_cast<cudaStream_t>(stream_) : b->stream;
    if (cudaError_t e = cudaMemsetAsync(b->d_rays, 0, 8, stream)) return cuda_fail(e, "pt_batch_render");
    const int strategy = b->strategy == PT_BATCH_AUTO ? PT_BATCH_ONE_LAUNCH : b->strategy;
    if (pt_status st = run_strategy(b, strategy, b->threads, stream)) return st;
    if (cudaError_t e = cudaEventRecord(b->done_event, stream)) return cuda_fail(e, "pt_batch_render");
    if (rays_out) {
        unsigned long long r = 0;
        if (cudaError_t e = cudaMemcpyAsync(&r, b->d_rays, 8, cudaMemcpyDeviceToHost, stream))
            return cuda_fail(e, "pt_batch_render: rays");
        if (cudaError_t e = cudaStreamSynchronize(stream)) return cuda_fail(e, "pt_batch_render");
        *rays_out = r;
    }
    return PT_OK;
}

pt_status pt_batch_output(const pt_batch* b, uint32_t i, const float** d_image) {
    clear_error();
    if (!b || !d_image || i >= b->scenes.size()) return fail(PT_ERR_INVALID_ARG, "pt_batch_output: bad argument");
    *d_image = b->d_out + b->scenes[i].out_offset;
    return PT_OK;
}

pt_status pt_batch_download(pt_batch* b, uint32_t i, float* host) {
    clear_error();
    if (!b || !host || i >= b->scenes.size()) return fail(PT_ERR_INVALID_ARG, "pt_batch_download: bad argument");
    if (cudaError_t e = cudaSetDevice(b->device)) return cuda_fail(e, "cudaSetDevice");
    const size_t floats = 3 * size_t(b->scenes[i].width) * b->scenes[i].height;
    // The last render may have run on a stream the caller passed, which the
    // copies below are not ordered against: wait for its end first.
    if (cudaError_t e = cudaEventSynchronize(b->done_event)) return cuda_fail(e, "pt_batch_download");
    if (cudaError_t e = cudaMemcpyAsync(host, b->d_out + b->scenes[i].out_offset, floats * 4, cudaMemcpyDeviceToHost,
                                        b->stream))
        return cuda_fail(e, "pt_batch_download");
    unsigned int st = 0;
    if (cudaError_t e = cudaMemcpyAsync(&st, b->d_status, 4, cudaMemcpyDeviceToHost, b->stream))
        return cuda_fail(e, "pt_batch_download: status");
    if (cudaError_t e = cudaStreamSynchronize(b->stream)) return cuda_fail(e, "pt_batch_download");
    if (st & PT_DEV_ERR_STACK) return fail(PT_ERR_STACK_OVERFLOW, "a traversal stack overflowed on the device");
    return PT_OK;
}

pt_status pt_batch_scene_times(pt_batch* b, double* ms) {
    clear_error();
    if (!b || !ms) return fail(PT_ERR_INVALID_ARG, "pt_batch_scene_times: null pointer");
    if (cudaError_t e = cudaSetDevice(b->device)) return cuda_fail(e, "cudaSetDevice");
    const size_t n = b->scenes.size();
    if (cudaError_t e = cudaEventSynchronize(b->done_event)) return cuda_fail(e, "pt_batch_scene_times");
    if (cudaError_t e = cudaStreamSynchronize(b->stream)) return cuda_fail(e, "pt_batch_scene_times");
    if (b->last_strategy == PT_BATCH_ONE_LAUNCH) {
        std::vector<unsigned long long> done(n);
        unsigned long long start = 0;
        cudaError_t e = cudaMemcpy(done.data(), b->d_done_ns, n * 8, cudaMemcpyDeviceToHost);
        if (!e) e = cudaMemcpy(&start, b->d_start, 8, cudaMemcpyDeviceToHost);
        if (e) return cuda_fail(e, "pt_batch_scene_times");
        for (size_t i = 0; i < n; ++i) ms[i] = done[i] >= start ? double(done[i] - start) * 1e-6 : 0.0;
    } else {
        for (size_t i = 0; i < n; ++i) {
            float t = 0;
            if (cudaError_t e = cudaEventElapsedTime(&t, b->start_event, b->scene_events[i]))
                return cuda_fail(e, "pt_batch_scene_times");
            ms[i] = t;
        }
    }
    return PT_OK;
}

pt_status pt_batch_get_info(const pt_batch* b, pt_batch_info* info) {
    clear_error();
    if (!b || !info) return fail(PT_ERR_INVALID_ARG, "pt_batch_get_info: null pointer");
    std::memset(info, 0, sizeof(*info));
    info->n_scenes = uint32_t(b->scenes.size());
    info->strategy = b->strategy == PT_BATCH_AUTO ? PT_BATCH_ONE_LAUNCH : b->strategy;
    info->threads = b->threads;
    info->tuned = b->tuned ? 1 : 0;
    info->total_pixels = b->total_pixels;
    info->total_samples = b->total_samples;
    info->device_bytes = b->arena_bytes;
    for (int k = 0; k < 8; ++k) info->tune_ms[k] = b->tune_ms[k];
    return PT_OK;
}

pt_status pt_batch_destroy(pt_batch* b) {
    if (!b) return PT_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto g : b->one_graph)
        if (g) cudaGraphExecDestroy(g);
    for (pt_scene* s : b->singles) pt_scene_destroy(s);
    for (cudaEvent_t e : b->scene_events) cudaEventDestroy(e);
    if (b->start_event) cudaEventDestroy(b->start_event);
    if (b->done_event) cudaEventDestroy(b->done_event);
    if (b->stream) cudaStreamDestroy(b->stream);
    if (b->arena) cudaFree(b->arena);
    delete b;
    return PT_OK;
}

}  // extern "C"
