// Batched rendering: many scenes of different size, resolution and spp in one
// persistent launch over one node arena.
//
// The scenes' arenas are merged on the host with every index rebased
// (batch.cpp), so the arena pointers are shared and a scene differs only by
// its tree roots, its ranges of large spheres and lights and its flags. Work
// items are the 8x4 tiles of all scenes' frames in scene order; a lane maps
// its item to a scene by binary search over the scenes' first items, builds
// that scene's view of the arena (a few registers) and renders the pixel
// exactly as the single-scene megakernel does -- same per-pixel stream,
// same order of sums, so each scene's image is bit-identical to rendering
// it alone. Each scene's completion time is taken from the global timer
// when its last pixel is written.
#include "batch.h"
#include "kernels.h"
#include "path.cuh"

using namespace ptd;

namespace {

constexpr int kTileW = 8, kTileH = 4;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Resident 128-thread blocks per SM the register allocation targets (scaled
// for other block sizes): 5 (at most 96 registers, as the megakernel). With
// the lane state in shared memory the 64-scene batch renders in 1,756 ms at 5
// against 1,847 ms at 4 (identical images); before it, 4 was best (3.42 s
// against 3.81 s at 3 and 3.60 s at 5).
#ifndef PT_BATCH_MIN_BLOCKS128
#define PT_BATCH_MIN_BLOCKS128 5
#endif

// Traversal-stack entries per lane in shared memory: 0, as measured best for
// the single-scene megakernel this kernel follows (at most 48 KB of static
// shared memory per block, so at most 12 entries at 256 threads).
#ifndef PT_BATCH_SH_STACK
#define PT_BATCH_SH_STACK 0
#endif

// Flat batches whose merged arena's leaves fit 8-byte stack entries
// (PtSceneDev::stack_pack8) walk with them, as the single-scene megakernel
// does for scenes larger than its threshold (the batch's scenes share one
// kernel; sphere-only scenes lose about 1% with it, mesh scenes gain 3-4%).
#ifndef PT_BATCH_PACK_STACK
#define PT_BATCH_PACK_STACK 1
#endif

#ifndef PT_BATCH_ONE_QUERY
#define PT_BATCH_ONE_QUERY 1
#endif

// As in the single-scene megakernel: each lane's pixel, sample number, scene
// number and running sum (which change once per path) in shared memory, the
// path itself too in the flat-scene form, and the per-scene frame values
// (size, spp, depth, seed) read from the scene table where they are used
// instead of held in registers for the whole loop.
#ifndef PT_BATCH_SMEM_STATE
#define PT_BATCH_SMEM_STATE 1
#endif

// Each scene's view of the merged arena (roots, large-sphere and light
// ranges, flags) prebuilt in global memory and referenced by the lane's scene
// number, instead of a copy patched per lane and held in registers.
#ifndef PT_BATCH_SCENE_VIEWS
#define PT_BATCH_SCENE_VIEWS 1
#endif

template <int THREADS, int TREES, bool TEX>
__global__ void __launch_bounds__(THREADS, PT_BATCH_MIN_BLOCKS128 * 128 / THREADS)
    batch_megakernel(PtSceneDev S0, PtBatchLaunch B) {
    // the stack in local memory, as the single-scene megakernel keeps it
    // (8-byte entries in the PT_TREES_FLAT8 form)
    PT_FORM_STACK(stack, TREES, THREADS, PT_BATCH_SH_STACK, 0);
    constexpr int QT = TREES == PT_TREES_FLAT8 ? int(PT_TREES_FLAT) : TREES;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) atomicMin(B.start_ns, global_ns());

    unsigned long long rays = 0;
    bool exhausted = false, has_pixel = false, in_path = false, overflow = false;
#if PT_BATCH_SMEM_STATE
    __shared__ int s_pix[4][THREADS];
    __shared__ V s_acc[THREADS];
    int& pi = s_pix[0][threadIdx.x];
    int& pj = s_pix[1][threadIdx.x];
    int& s = s_pix[2][threadIdx.x];
    int& sci = s_pix[3][threadIdx.x];
    V& acc = s_acc[threadIdx.x];
    pi = pj = s = sci = 0;
    acc = mk(0, 0, 0);
    constexpr bool SMEM_PATH = QT == PT_TREES_FLAT;
#else
    int pi = 0, pj = 0, s = 0, sci = 0;
    V acc = mk(0, 0, 0);
    constexpr bool SMEM_PATH = false;
#endif
    __shared__ Path s_path[SMEM_PATH ? THREADS : 1];
    Path local_path;
    Path& path = SMEM_PATH ? s_path[threadIdx.x] : local_path;
    First first = {mk(0, 0, 0), mk(0, 0, 0)};
    Sampler smp;
    Rng rng;
#if !PT_BATCH_SCENE_VIEWS
    PtSceneDev S = S0;
#endif
    // Scenes without instances: one ray query per trip, the pending shadow
    // rays in shared memory (as in the single-scene megakernel).
    constexpr bool ONE_QUERY = PT_BATCH_ONE_QUERY && QT == PT_TREES_FLAT;
    __shared__ float pend[10][ONE_QUERY ? THREADS : 1];
    bool shadow_pending = false, done_after_shadow = false;

    while (true) {
        const bool need = !has_pixel && !exhausted;
        const unsigned want = __ballot_sync(0xffffffffu, need);
        if (want) {
            const int leader = __ffs(want) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(B.work, uint32_t(__popc(want)));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                const uint32_t item = base + __popc(want & ((1u << lane) - 1u));
                if (item >= B.total_items) {
                    exhausted = true;
                } else {
                    // The scene whose items contain this one.
                    uint32_t lo = 0, hi = B.n_scenes - 1;
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi + 1) >> 1;
                        if (__ldg(&B.scenes[mid].item_base) <= item) lo = mid;
                        else hi = mid - 1;
                    }
                    sci = int(lo);
                    const PtBatchScene& D = B.scenes[lo];
                    const uint32_t local = item - __ldg(&D.item_base);
                    const uint32_t tx = __ldg(&D.tiles_x);
                    const int width = int(__ldg(&D.width)), height = int(__ldg(&D.height));
                    const uint32_t tile = local >> 5, l = local & 31u;
                    pi = int((tile % tx) * kTileW + (l & 7u));
                    pj = int((tile / tx) * kTileH + (l >> 3));
                    if (pi < width && pj < height) {
                        has_pixel = true;
                        s = 0;
                        in_path = false;
                        acc = mk(0, 0, 0);
#if !PT_BATCH_SCENE_VIEWS
                        S.flat_root = __ldg(&D.flat_root);
                        S.inst_root = __ldg(&D.inst_root);
                        S.large = S0.large + __ldg(&D.large_base);
                        S.large_mat = S0.large_mat + __ldg(&D.large_base);
                        S.n_large = __ldg(&D.n_large);
                        S.lights = S0.lights + __ldg(&D.light_base);
                        S.n_lights = __ldg(&D.n_lights);
                        S.sky = int(__ldg(&D.sky));
                        S.sample_lights = int(__ldg(&D.sample_lights));
#endif
                    }
                }
            }
        }
        if (__all_sync(0xffffffffu, exhausted)) break;
        if (!has_pixel) continue;

        const PtBatchScene& D = B.scenes[sci];
#if PT_BATCH_SCENE_VIEWS
        const PtSceneDev& S = B.views[sci];
#endif
        if (!in_path) {
            if (int(__ldg(&D.depth)) <= 0) {
                s = int(__ldg(&D.spp));
            } else {
                const uint32_t idx = uint32_t(s);
                const uint64_t seed = __ldg(&D.seed);
                smp.begin(seed, pi, pj, idx);
                float du, dv;
                smp.sample_2d(0, rng, du, dv);
                const float u = (float(pi) + du) / float(int(__ldg(&D.width)) - 1);
                const float v = (float(pj) + dv) / float(int(__ldg(&D.height)) - 1);
                const V origin = mk(__ldg(&D.cam[0]), __ldg(&D.cam[1]), __ldg(&D.cam[2]));
                const V llc = mk(__ldg(&D.cam[3]), __ldg(&D.cam[4]), __ldg(&D.cam[5]));
                const V hor = mk(__ldg(&D.cam[6]), __ldg(&D.cam[7]), __ldg(&D.cam[8]));
                const V ver = mk(__ldg(&D.cam[9]), __ldg(&D.cam[10]), __ldg(&D.cam[11]));
                path.o = origin;
                path.d = llc + hor * u + ver * v - origin;
                path.tp = mk(1, 1, 1);
                path.rad = mk(0, 0, 0);
                path.bounce = 0;
                path.sampled = false;
                path.mis_pdf = 0;
                rng.seed(sample_stream_seed(seed, pi, pj, idx));
                in_path = true;
            }
        }

        if constexpr (ONE_QUERY) {
            if (in_path && query_trip<false, TEX, false>(S, path, int(__ldg(&D.depth)), smp, rng, first, pend,
                                                         shadow_pending,
                                                  done_after_shadow, stack, rays, overflow)) {
                acc = acc + path.rad;
                in_path = false;
                ++s;
            }
        } else if (in_path) {
            ++rays;
            smp.set_bounce(path.bounce);
            float t = 1000.0f;
            Hit h;
            Counts cnt;
            Rec rec;
            if (!closest<false, QT>(S, path.o, path.d, 0.001f, t, h, stack, cnt)) {
                overflow = true;
                h.kind = PT_HIT_NONE;
            }
            const bool hit = h.kind != PT_HIT_NONE;
            if (hit) fill<TEX, false>(S, h, path.o, path.d, t, rec);
            bool nee;
            Shadow sh;
            const int step = shade<false, TEX, false>(S, path, hit, rec, int(__ldg(&D.depth)), smp, rng, first, nee, sh,
                                                      rays);
            if (nee) {
                bool ovf = false;
                if (!occluded<false, QT>(S, sh.o, sh.d, 0.001f, sh.t_max, stack, cnt, &ovf)) path.rad = path.rad + sh.value;
                overflow |= ovf;
            }
            if (step == STEP_DONE) {
                acc = acc + path.rad;
                in_path = false;
                ++s;
            }
        }

        const int spp = int(__ldg(&D.spp));
        if (s >= spp) {
            const int width = int(__ldg(&D.width)), height = int(__ldg(&D.height));
            const uint32_t sc = uint32_t(sci);
            const float scale = 1.0f / float(spp);
            float* out = B.out + __ldg(&D.out_offset) + 3 * (size_t(height - 1 - pj) * width + pi);
            out[0] = acc.x * scale;
            out[1] = acc.y * scale;
            out[2] = acc.z * scale;
            has_pixel = false;
            const uint32_t px = uint32_t(width) * uint32_t(height);
            if (atomicAdd(B.done_pixels + sc, 1u) == px - 1) B.done_ns[sc] = global_ns();
        }
    }
    unsigned long long total = rays;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) total += __shfl_down_sync(0xffffffffu, total, off);
    if (lane == 0 && B.rays) atomicAdd(B.rays, total);
    if (__any_sync(0xffffffffu, overflow) && lane == 0) atomicOr(S0.status, PT_DEV_ERR_STACK);
}

template <int THREADS, int TREES, bool TEX>
void launch(const PtSceneDev& S, const PtBatchLaunch& b, int sms, cudaStream_t stream) {
    const int blocks =
        pt_resident_blocks(reinterpret_cast<const void*>(batch_megakernel<THREADS, TREES, TEX>), THREADS, 0);
    batch_megakernel<THREADS, TREES, TEX><<<sms * blocks, THREADS, 0, stream>>>(S, b);
}

template <int TREES, bool TEX>
void launch_threads(const PtSceneDev& S, const PtBatchLaunch& b, int threads, int sms, cudaStream_t stream) {
    switch (threads) {
        case 64:
            launch<64, TREES, TEX>(S, b, sms, stream);
            break;
        case 256:
            launch<256, TREES, TEX>(S, b, sms, stream);
            break;
        default:
            launch<128, TREES, TEX>(S, b, sms, stream);
            break;
    }
}

}  // namespace

// The single-loop traversal when some scene has instances, one loop per tree
// otherwise (with 8-byte stack entries where they fit); texture code only
// when some scene has textures.
cudaError_t pt_launch_batch(const PtSceneDev& S, const PtBatchLaunch& b, int threads, int sms, cudaStream_t stream) {
    if (S.has_textures) {
        if (b.any_instances)
            launch_threads<PT_TREES_ONE, true>(S, b, threads, sms, stream);
        else
            launch_threads<PT_TREES_FLAT, true>(S, b, threads, sms, stream);
    } else if (b.any_instances) {
        launch_threads<PT_TREES_ONE, false>(S, b, threads, sms, stream);
    } else if (PT_BATCH_PACK_STACK && S.stack_pack8) {
        launch_threads<PT_TREES_FLAT8, false>(S, b, threads, sms, stream);
    } else {
        launch_threads<PT_TREES_FLAT, false>(S, b, threads, sms, stream);
    }
    return cudaGetLastError();
}
