// Persistent-thread megakernel path tracer.
//
// The CPU renderer gives each thread a whole scanline, taken from an atomic
// row counter (src/main.cpp:137-158), and runs samples_per_pixel paths per
// pixel one after another (include/renderer.hpp:366-409). Here each LANE owns
// a pixel, runs its samples one path after another (so the per-pixel sums
// are formed in the same order as the reference's), and advances one bounce
// (or, for scenes without instances, one ray query) per loop trip; when its pixel is finished it takes the next from a global
// counter, warp-aggregated (one atomicAdd per warp per refill). Pixels are
// numbered by 8x4 tiles so a warp's first pixels are neighbours and their
// primary rays coherent. Work per warp is therefore balanced at path
// granularity and no lane waits for another lane's pixel.
#include "kernels.h"
#include "path.cuh"

using namespace ptd;

namespace {

constexpr int kTileW = 8, kTileH = 4;

// Resident 128-thread blocks per SM the register allocation targets (5: at
// most 96 registers; +6.6% on the 1024x1024 room frame and +8% on the
// 10,000-instance frame against 3 and 4, which the compiler met with 116-128
// registers; 6 lost).
#ifndef PT_MEGA_MIN_BLOCKS
#define PT_MEGA_MIN_BLOCKS 5
#endif

// The pixel coordinates, sample number and running sum of each lane in
// shared memory instead of registers (they change once per path): 170 -> 100
// bytes of spills in the flat-scene form, room frame +0.8%, images identical.
#ifndef PT_MEGA_SMEM_STATE
#define PT_MEGA_SMEM_STATE 1
#endif

// The path state of each lane in shared memory too, in the flat-scene form:
// no spills left there, room frame +1.0%, random spheres +3.7%; the instanced
// form lost 3% with it and keeps registers (the RNG state moved as well
// gained nothing more).
#ifndef PT_MEGA_SMEM_PATH
#define PT_MEGA_SMEM_PATH 1
#endif

// Scenes without instances trace one query per loop trip (a path ray or a
// shadow ray) through one traversal call site: lanes on shadow rays traverse
// alongside lanes on path rays instead of after them. Same images; +28.6% on
// the 1920x1080x16 random-spheres frame (2,797 -> 3,597 Mrays/s), the room
// frame within 0.5%, and at four blocks per SM 7% slower.
#ifndef PT_MEGA_ONE_QUERY
#define PT_MEGA_ONE_QUERY 1
#endif

// Traversal-stack entries per lane in shared memory (the rest in its local
// array). Measured on the 1024x1024 room frame, the 1080p random-spheres
// frame and the 10,000-instance frame (identical images): 0 is fastest; 2, 4
// and 8 entries lost 1-3%, 1-5% and 1-6% (the kernel already keeps 15 KB of
// path state per block in shared memory; a stack on top leaves the SM's L1
// data cache 60 KB smaller for node and primitive fetches), 16 lost 14%.
// The wavefront stages and ray-query kernels, with no other shared state,
// gain from it and use PT_SH_STACK.
#ifndef PT_MEGA_SH_STACK
#define PT_MEGA_SH_STACK 0
#endif

// A second flat-scene form whose stack has 8-byte entries (PackedStack,
// PT_TREES_FLAT8), launched for flat scenes whose leaves fit them
// (PtSceneDev::stack_pack8) and whose nodes and leaf slots take more than
// PT_MEGA_PACK_MIN_KIB: the deep local array is 768 instead of 1,536 bytes
// per lane, and its hot entries take half the L1 lines. Measured on one
// B200 with identical images (Mrays/s, 16-byte -> 8-byte): room frames with
// the icosphere at 1,290 / 5,130 / 20,490 / 81,930 triangles (1024x1024,
// 16 spp; about 0.1, 0.4, 1.8, 7 MB of nodes and slots) 3,191 -> 3,325 /
// 2,921 -> 3,030 / 2,737 -> 2,827 / 2,586 -> 2,661 (+4.2 / +3.7 / +3.3 /
// +2.9%), the 64-spp bench frame 2,608 -> 2,684; the 1080p random spheres
// (488 spheres, about 44 KB) 4,210 -> 4,191 and 4,222 -> 4,165 in two runs
// (-0.5 / -1.3%: the packing instructions without an L1 gain), hence the
// threshold between the two. Shared-memory entries on top
// (PT_MEGA_SH_STACK8 = 4, 8, 12: 4, 8, 12 KB per block) lost 4-6% on the
// room and random-spheres frames.
#ifndef PT_MEGA_PACK_STACK
#define PT_MEGA_PACK_STACK 1
#endif
#ifndef PT_MEGA_PACK_MIN_KIB
#define PT_MEGA_PACK_MIN_KIB 64
#endif
#ifndef PT_MEGA_SH_STACK8
#define PT_MEGA_SH_STACK8 0
#endif


// EXT: the extended light sampling of PT_FLAG_NEE_EXTENDED (production
// streams only); false compiles exactly the reference's estimator.
template <bool AUX, bool SNAP, int TREES, bool TEX, bool EXT>
__global__ void __launch_bounds__(128, PT_MEGA_MIN_BLOCKS) megakernel(PtSceneDev S, PtRenderParams P, uint32_t tiles_x,
                                                  uint32_t total_items) {
    PT_FORM_STACK(stack, TREES, 128, PT_MEGA_SH_STACK, PT_MEGA_SH_STACK8);
    // the traversal form the queries compile (PT_TREES_FLAT8 is the flat one
    // with the other stack)
    constexpr int QT = TREES == PT_TREES_FLAT8 ? int(PT_TREES_FLAT) : TREES;
    const int lane = threadIdx.x & 31;
    const Cam cam = {mk(P.cam.origin[0], P.cam.origin[1], P.cam.origin[2]),
                     mk(P.cam.llc[0], P.cam.llc[1], P.cam.llc[2]),
                     mk(P.cam.horizontal[0], P.cam.horizontal[1], P.cam.horizontal[2]),
                     mk(P.cam.vertical[0], P.cam.vertical[1], P.cam.vertical[2])};
    const float scale = 1.0f / float(P.spp);
    const float wm1 = float(P.width - 1), hm1 = float(P.height - 1);

    unsigned long long rays = 0;
    bool exhausted = false, has_pixel = false, in_path = false;
#if PT_MEGA_SMEM_STATE
    // The pixel, its sample number and its running sum change once per
    // path: they live in shared memory, leaving registers to the traversal.
    __shared__ int s_pix[3][128];
    __shared__ V s_acc[128];
    int& pi = s_pix[0][threadIdx.x];
    int& pj = s_pix[1][threadIdx.x];
    int& s = s_pix[2][threadIdx.x];
    V& acc = s_acc[threadIdx.x];
    pi = pj = s = 0;
    acc = mk(0, 0, 0);
    V acc_albedo = mk(0, 0, 0), acc_normal = mk(0, 0, 0);
#else
    int pi = 0, pj = 0, s = 0;
    V acc = mk(0, 0, 0), acc_albedo = mk(0, 0, 0), acc_normal = mk(0, 0, 0);
#endif
    float lum2 = 0;
    // Flat-scene form: the path (ray, throughput, radiance, bounce) in shared
    // memory too, read into registers where a query or shading needs it.
    constexpr bool SMEM_PATH = PT_MEGA_SMEM_PATH && QT == PT_TREES_FLAT;
    __shared__ Path s_path[SMEM_PATH ? 128 : 1];
    Path local_path;
    Path& path = SMEM_PATH ? s_path[threadIdx.x] : local_path;
    First first = {mk(0, 0, 0), mk(0, 0, 0)};
    Sampler smp;
    Rng rng;
    bool overflow = false;
    // Single-query form: the pending shadow ray (origin, direction, t_max,
    // unblocked value) of each lane, kept in shared memory between trips.
    constexpr bool ONE_QUERY = PT_MEGA_ONE_QUERY && QT == PT_TREES_FLAT;
    __shared__ float pend[10][ONE_QUERY ? 128 : 1];
    bool shadow_pending = false, done_after_shadow = false;

    while (true) {
        // Refill lanes without a pixel.
        const bool need = !has_pixel && !exhausted;
        const unsigned want = __ballot_sync(0xffffffffu, need);
        if (want) {
            const int leader = __ffs(want) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(P.work, uint32_t(__popc(want)));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                const uint32_t item = base + __popc(want & ((1u << lane) - 1u));
                if (item >= total_items) {
                    exhausted = true;
                } else {
                    const uint32_t tile = item >> 5, l = item & 31u;
                    pi = int((tile % tiles_x) * kTileW + (l & 7u));
                    pj = P.row0 + int((tile / tiles_x) * kTileH + (l >> 3));
                    if (pi < P.width && pj < P.row0 + P.rows) {
                        has_pixel = true;
                        s = 0;
                        in_path = false;
                        acc = acc_albedo = acc_normal = mk(0, 0, 0);
                        lum2 = 0;
                    }
                }
            }
        }
        if (__all_sync(0xffffffffu, exhausted)) break;
        if (!has_pixel) continue;

        if (!in_path) {
            if (P.depth <= 0 || P.spp <= 0) {
                s = P.spp;  // nothing to trace: every sample is black
            } else {
                // render_row_impl's sample loop body (:379-385)
                const uint32_t idx = uint32_t(P.first_sample + s);
                smp.begin(P.seed, pi, pj, idx);
                float du, dv;
                smp.sample_2d(0, rng, du, dv);
                const float u = (float(pi) + du) / wm1;
                const float v = (float(pj) + dv) / hm1;
                path.o = cam.origin;
                path.d = cam.llc + cam.horizontal * u + cam.vertical * v - cam.origin;
                path.tp = mk(1, 1, 1);
                path.rad = mk(0, 0, 0);
                path.bounce = 0;
                path.sampled = false;
                path.mis_pdf = 0;
                first = {mk(0, 0, 0), mk(0, 0, 0)};
                if (SNAP) {
                    const uint64_t* st = P.states + 4 * ((size_t(pj) * P.width + pi) * P.spp + s);
                    rng.s0 = st[0];
                    rng.s1 = st[1];
                    rng.s2 = st[2];
                    rng.s3 = st[3];
                } else {
                    rng.seed(sample_stream_seed(P.seed, pi, pj, idx));
                }
                in_path = true;
            }
        }

        if constexpr (ONE_QUERY) {
            if (in_path && query_trip<AUX, TEX, EXT>(S, path, P.depth, smp, rng, first, pend, shadow_pending,
                                                done_after_shadow, stack, rays, overflow)) {
                acc = acc + path.rad;
                if (AUX) {
                    acc_albedo = acc_albedo + first.albedo;
                    acc_normal = acc_normal + first.normal;
                    const float l = luminance(path.rad);
                    lum2 += l * l;
                }
                in_path = false;
                ++s;
            }
        } else if (in_path) {
            // One iteration of ray_color's bounce loop.
            ++rays;
            smp.set_bounce(path.bounce);
            float t = 1000.0f;
            Hit h;
            Counts cnt;
            Rec rec;
            bool ok = closest<false, QT>(S, path.o, path.d, 0.001f, t, h, stack, cnt);
            if (!ok) {
                overflow = true;
                h.kind = PT_HIT_NONE;
            }
            const bool hit = h.kind != PT_HIT_NONE;
            if (hit) fill<TEX, EXT>(S, h, path.o, path.d, t, rec);
            bool nee;
            Shadow sh;
            const int step = shade<AUX, TEX, EXT>(S, path, hit, rec, P.depth, smp, rng, first, nee, sh, rays);
            if (nee) {
                bool ovf = false;
                if (!occluded<false, QT>(S, sh.o, sh.d, 0.001f, sh.t_max, stack, cnt, &ovf))
                    path.rad = path.rad + sh.value;
                overflow |= ovf;
            }
            if (step == STEP_DONE) {
                acc = acc + path.rad;
                if (AUX) {
                    acc_albedo = acc_albedo + first.albedo;
                    acc_normal = acc_normal + first.normal;
                    const float l = luminance(path.rad);
                    lum2 += l * l;
                }
                in_path = false;
                ++s;
            }
        }

        if (s >= P.spp) {
            const int row = P.flip ? (P.height - 1 - pj) : (pj - P.row0);
            const size_t px = size_t(row) * P.width + pi;
            P.out[3 * px + 0] = acc.x * scale;
            P.out[3 * px + 1] = acc.y * scale;
            P.out[3 * px + 2] = acc.z * scale;
            if (AUX) {
                float* a = P.aux + 7 * px;
                a[0] = acc_albedo.x * scale;
                a[1] = acc_albedo.y * scale;
                a[2] = acc_albedo.z * scale;
                a[3] = acc_normal.x * scale;
                a[4] = acc_normal.y * scale;
                a[5] = acc_normal.z * scale;
                a[6] = lum2 * scale;
            }
            has_pixel = false;
        }
    }

    // Ray count: warp sum, one atomic per warp.
    unsigned long long total = rays;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) total += __shfl_down_sync(0xffffffffu, total, off);
    if (lane == 0 && P.rays) atomicAdd(P.rays, total);
    if (__any_sync(0xffffffffu, overflow) && lane == 0) atomicOr(S.status, PT_DEV_ERR_STACK);
}

template <bool AUX, bool SNAP, int TREES, bool TEX, bool EXT>
cudaError_t launch(const PtSceneDev& S, const PtRenderParams& p, const PtLaunchShape& shape, cudaStream_t stream) {
    const uint32_t tiles_x = uint32_t((p.width + kTileW - 1) / kTileW);
    const uint32_t tiles_y = uint32_t((p.rows + kTileH - 1) / kTileH);
    const uint32_t total = tiles_x * tiles_y * 32u;
    megakernel<AUX, SNAP, TREES, TEX, EXT><<<shape.blocks, shape.threads, 0, stream>>>(S, p, tiles_x, total);
    return cudaGetLastError();
}

template <int TREES, bool TEX>
cudaError_t launch_form(const PtSceneDev& S, const PtRenderParams& p, const PtLaunchShape& shape,
                        cudaStream_t stream) {
    const bool aux = p.aux != nullptr, snap = p.rng_mode == 1;
    if (p.nee_ext)  // production streams only (the host refuses it with snapshots)
        return aux ? launch<true, false, TREES, TEX, true>(S, p, shape, stream)
                   : launch<false, false, TREES, TEX, true>(S, p, shape, stream);
    if (aux)
        return snap ? launch<true, true, TREES, TEX, false>(S, p, shape, stream)
                    : launch<true, false, TREES, TEX, false>(S, p, shape, stream);
    return snap ? launch<false, true, TREES, TEX, false>(S, p, shape, stream)
                : launch<false, false, TREES, TEX, false>(S, p, shape, stream);
}

template <int TREES, bool TEX>
int occupancy(int threads, bool aux, bool snap, bool ext) {
    const void* fn = ext ? (aux ? reinterpret_cast<const void*>(megakernel<true, false, TREES, TEX, true>)
                                : reinterpret_cast<const void*>(megakernel<false, false, TREES, TEX, true>))
                   : aux ? (snap ? reinterpret_cast<const void*>(megakernel<true, true, TREES, TEX, false>)
                                 : reinterpret_cast<const void*>(megakernel<true, false, TREES, TEX, false>))
                         : (snap ? reinterpret_cast<const void*>(megakernel<false, true, TREES, TEX, false>)
                                 : reinterpret_cast<const void*>(megakernel<false, false, TREES, TEX, false>));
    return pt_resident_blocks(fn, threads, 0);
}

// The single-loop traversal for scenes with instances, one loop per tree
// otherwise; texture code only in the kernels for scenes with textures; for
// large flat scenes without textures whose leaves fit them, 8-byte stack
// entries.
bool one_loop(const PtSceneDev& S) { return S.use_bvh && S.inst_root != PT_NONE; }
bool flat_only(const PtSceneDev& S) { return S.inst_root == PT_NONE && S.n_instances == 0; }
bool flat8(const PtSceneDev& S) {
    return PT_MEGA_PACK_STACK && S.use_bvh && S.stack_pack8 && S.tree_kib > PT_MEGA_PACK_MIN_KIB;
}

}  // namespace

cudaError_t pt_launch_megakernel(const PtSceneDev& S, const PtRenderParams& p, const PtLaunchShape& shape,
                                 cudaStream_t stream) {
    if (S.has_textures)
        return one_loop(S)   ? launch_form<PT_TREES_ONE, true>(S, p, shape, stream)
               : flat_only(S) ? launch_form<PT_TREES_FLAT, true>(S, p, shape, stream)
                              : launch_form<PT_TREES_EACH, true>(S, p, shape, stream);
    if (one_loop(S)) return launch_form<PT_TREES_ONE, false>(S, p, shape, stream);
    if (!flat_only(S)) return launch_form<PT_TREES_EACH, false>(S, p, shape, stream);
    return flat8(S) ? launch_form<PT_TREES_FLAT8, false>(S, p, shape, stream)
                    : launch_form<PT_TREES_FLAT, false>(S, p, shape, stream);
}

int pt_megakernel_blocks_per_sm(const PtSceneDev& S, int threads, bool aux, bool snapshot, bool ext) {
    if (S.has_textures)
        return one_loop(S)   ? occupancy<PT_TREES_ONE, true>(threads, aux, snapshot, ext)
               : flat_only(S) ? occupancy<PT_TREES_FLAT, true>(threads, aux, snapshot, ext)
                              : occupancy<PT_TREES_EACH, true>(threads, aux, snapshot, ext);
    if (one_loop(S)) return occupancy<PT_TREES_ONE, false>(threads, aux, snapshot, ext);
    if (!flat_only(S)) return occupancy<PT_TREES_EACH, false>(threads, aux, snapshot, ext);
    return flat8(S) ? occupancy<PT_TREES_FLAT8, false>(threads, aux, snapshot, ext)
                    : occupancy<PT_TREES_FLAT, false>(threads, aux, snapshot, ext);
}
