// Wavefront path tracer: the same integrator as the megakernel, split into
// stages that each run over a queue of path slots:
//
//   extend  closest hit for every slot in the current ray queue
//   shade   the rest of the bounce (emission, scatter, light sample, Russian
//           roulette); pushes the slot to the shadow queue when it made a
//           shadow ray, to the next ray queue when the path goes on, and
//           starts the slot's next sample (or next pixel) when the path ended
//   shadow  any hit for every shadow ray; adds the light sample when it is
//           not blocked, and finishes paths that ended waiting for it
//
// A slot owns one pixel at a time and runs its samples one after another, as
// a megakernel lane does, so per-pixel sums are formed in the same order and
// the image is bit-identical to the megakernel's. Queues are compacted with
// warp ballots: one atomicAdd per warp, each lane writing at its rank.
// The traversal-heavy extend/shadow kernels carry only the ray and hit, so
// they run at lower register counts (higher occupancy) than the megakernel.
#include "wavefront.h"
#include "path.cuh"

using namespace ptd;

namespace {

constexpr int kTileW = 8, kTileH = 4;
constexpr uint32_t F_IN_PATH = 1u << 8, F_SAMPLED = 1u << 9, F_DONE_PENDING = 1u << 10, F_HAS_PIXEL = 1u << 11;

struct WfView {  // device pointers into the scratch arena
    float4 *ray_o, *ray_d, *tp, *rad, *acc, *acc_albedo, *acc_normal, *first_albedo, *first_normal, *sh_d, *sh_v;
    uint4* meta;    // (item, sample, bounce | flags, pixel_seed)
    ulonglong2* rng;  // 2 per slot
    uint4* hit;     // (kind, index, inst, t bits)
    float2* huv;
    uint32_t* queue[2];
    uint32_t* shadow_q;
    uint32_t* counts;  // [0], [1]: ray queues, [2]: shadow queue, [3]: pixel work counter, [4]: live slots
    uint32_t slots;
};

// Warp-ballot compaction: the lanes that want to push agree on a count, one
// lane reserves that many entries, and each writes at its rank. The set of
// participating lanes is taken once, so the ballot and the broadcast agree.
__device__ __forceinline__ void push(uint32_t* queue, uint32_t* count, bool want, uint32_t value) {
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, want);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, uint32_t(__popc(mask)));
    base = __shfl_sync(active, base, leader);
    if (want) queue[base + __popc(mask & ((1u << lane) - 1u))] = value;
}

struct Frame {
    PtRenderParams P;
    uint32_t tiles_x, total_items;
    Cam cam;
};

__device__ __forceinline__ void pixel_of(const Frame& F, uint32_t item, int& pi, int& pj, bool& valid) {
    const uint32_t tile = item >> 5, l = item & 31u;
    pi = int((tile % F.tiles_x) * kTileW + (l & 7u));
    pj = F.P.row0 + int((tile / F.tiles_x) * kTileH + (l >> 3));
    valid = pi < F.P.width && pj < F.P.row0 + F.P.rows;
}

// Starts sample `s` of the slot's pixel: camera ray, sampler, random stream.
__device__ __forceinline__ void start_sample(const Frame& F, const WfView& W, uint32_t slot, uint32_t item, int pi,
                                             int pj, uint32_t s) {
    const PtRenderParams& P = F.P;
    const uint32_t idx = uint32_t(P.first_sample) + s;
    Sampler smp;
    smp.begin(P.seed, pi, pj, idx);
    Rng rng;
    float du, dv;
    smp.sample_2d(0, rng, du, dv);
    const float u = (float(pi) + du) / float(P.width - 1);
    const float v = (float(pj) + dv) / float(P.height - 1);
    const V d = F.cam.llc + F.cam.horizontal * u + F.cam.vertical * v - F.cam.origin;
    if (P.rng_mode == PT_RNG_SNAPSHOT) {
        const uint64_t* st = P.states + 4 * ((size_t(pj) * P.width + pi) * P.spp + s);
        rng.s0 = st[0];
        rng.s1 = st[1];
        rng.s2 = st[2];
        rng.s3 = st[3];
    } else {
        rng.seed(sample_stream_seed(P.seed, pi, pj, idx));
    }
    W.ray_o[slot] = make_float4(F.cam.origin.x, F.cam.origin.y, F.cam.origin.z, 0);
    W.ray_d[slot] = make_float4(d.x, d.y, d.z, 0);
    W.tp[slot] = make_float4(1, 1, 1, 0);
    W.rad[slot] = make_float4(0, 0, 0, 0);
    W.first_albedo[slot] = make_float4(0, 0, 0, 0);
    W.first_normal[slot] = make_float4(0, 0, 0, 0);
    W.rng[2 * slot] = make_ulonglong2(rng.s0, rng.s1);
    W.rng[2 * slot + 1] = make_ulonglong2(rng.s2, rng.s3);
    W.meta[slot] = make_uint4(item, s, F_IN_PATH | F_HAS_PIXEL, smp.pixel_seed);
}

// Writes the pixel's averages.
template <bool AUX>
__device__ __forceinline__ void write_pixel(const Frame& F, const WfView& W, uint32_t slot, int pi, int pj) {
    const PtRenderParams& P = F.P;
    const float scale = 1.0f / float(P.spp);
    const int row = P.flip ? (P.height - 1 - pj) : (pj - P.row0);
    const size_t px = size_t(row) * P.width + pi;
    const float4 a = W.acc[slot];
    P.out[3 * px + 0] = a.x * scale;
    P.out[3 * px + 1] = a.y * scale;
    P.out[3 * px + 2] = a.z * scale;
    if (AUX) {
        const float4 al = W.acc_albedo[slot], nm = W.acc_normal[slot];
        float* x = P.aux + 7 * px;
        x[0] = al.x * scale;
        x[1] = al.y * scale;
        x[2] = al.z * scale;
        x[3] = nm.x * scale;
        x[4] = nm.y * scale;
        x[5] = nm.z * scale;
        x[6] = a.w * scale;
    }
}

// Takes pixels from the work counter until one is valid; returns false when
// the frame is exhausted. One atomic per slot refill (refills are spread out
// over the frame, unlike the megakernel's lock-step warps).
__device__ __forceinline__ bool next_pixel(const Frame& F, const WfView& W, uint32_t& item, int& pi, int& pj) {
    while (true) {
        item = atomicAdd(&W.counts[3], 1u);
        if (item >= F.total_items) return false;
        bool valid;
        pixel_of(F, item, pi, pj, valid);
        if (valid) return true;
    }
}

// The slot's sample ended with radiance rad: accumulate, then start the next
// sample or pixel. Returns true if the slot has a new path to trace.
template <bool AUX>
__device__ __forceinline__ bool finish_sample(const Frame& F, const WfView& W, uint32_t slot) {
    const uint4 m = W.meta[slot];
    const float4 r = W.rad[slot];
    float4 a = W.acc[slot];
    a.x = a.x + r.x;
    a.y = a.y + r.y;
    a.z = a.z + r.z;
    if (AUX) {
        const float l = luminance(mk(r.x, r.y, r.z));
        a.w += l * l;
        const float4 fa = W.first_albedo[slot], fn = W.first_normal[slot];
        float4 al = W.acc_albedo[slot], nm = W.acc_normal[slot];
        al.x = al.x + fa.x;
        al.y = al.y + fa.y;
        al.z = al.z + fa.z;
        nm.x = nm.x + fn.x;
        nm.y = nm.y + fn.y;
        nm.z = nm.z + fn.z;
        W.acc_albedo[slot] = al;
        W.acc_normal[slot] = nm;
    }
    W.acc[slot] = a;
    uint32_t item = m.x;
    int pi, pj;
    bool valid;
    pixel_of(F, item, pi, pj, valid);
    const uint32_t s = m.y + 1;
    if (s < uint32_t(F.P.spp)) {
        start_sample(F, W, slot, item, pi, pj, s);
        return true;
    }
    write_pixel<AUX>(F, W, slot, pi, pj);
    if (!next_pixel(F, W, item, pi, pj)) {
        W.meta[slot] = make_uint4(0, 0, 0, 0);
        return false;
    }
    W.acc[slot] = make_float4(0, 0, 0, 0);
    W.acc_albedo[slot] = make_float4(0, 0, 0, 0);
    W.acc_normal[slot] = make_float4(0, 0, 0, 0);
    start_sample(F, W, slot, item, pi, pj, 0);
    return true;
}

// Every slot takes a first pixel and starts its first sample.
template <bool AUX>
__global__ void __launch_bounds__(256) wf_init(Frame F, WfView W) {
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < W.slots; slot += gridDim.x * blockDim.x) {
        uint32_t item;
        int pi, pj;
        const bool got = next_pixel(F, W, item, pi, pj);
        if (got) {
            W.acc[slot] = make_float4(0, 0, 0, 0);
            W.acc_albedo[slot] = make_float4(0, 0, 0, 0);
            W.acc_normal[slot] = make_float4(0, 0, 0, 0);
            if (F.P.depth <= 0) {
                // Nothing to trace: every sample is black; write at once and
                // take the next pixel until the frame is exhausted.
                do {
                    write_pixel<AUX>(F, W, slot, pi, pj);
                } while (next_pixel(F, W, item, pi, pj));
                W.meta[slot] = make_uint4(0, 0, 0, 0);
            } else {
                start_sample(F, W, slot, item, pi, pj, 0);
            }
        } else {
            W.meta[slot] = make_uint4(0, 0, 0, 0);
        }
        push(W.queue[0], &W.counts[0], got && F.P.depth > 0, slot);
    }
}

// Closest hit for each queued ray.
__global__ void __launch_bounds__(128) wf_extend(PtSceneDev S, WfView W, int cur) {
    PT_TRAV_STACK(stack, 128);
    const uint32_t n = W.counts[cur];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        W.counts[cur ^ 1] = 0;  // the next ray queue and the shadow queue start empty
        W.counts[2] = 0;
    }
    bool overflow = false;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t slot = W.queue[cur][q];
        const float4 o = W.ray_o[slot], d = W.ray_d[slot];
        float t = 1000.0f;
        Hit h;
        Counts cnt;
        if (!closest<false>(S, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), 0.001f, t, h, stack, cnt)) {
            overflow = true;
            h.kind = PT_HIT_NONE;
        }
        W.hit[slot] = make_uint4(h.kind, h.index, h.inst, __float_as_uint(t));
        W.huv[slot] = make_float2(h.u, h.v);
    }
    if (overflow) atomicOr(S.status, PT_DEV_ERR_STACK);
}

// The rest of the bounce for each queued ray.
template <bool AUX>
__global__ void __launch_bounds__(128) wf_shade(PtSceneDev S, Frame F, WfView W, int cur,
                                                unsigned long long* rays_out) {
    const uint32_t n = W.counts[cur];
    const int nxt = cur ^ 1;
    unsigned long long rays = 0;
    const uint32_t n_round = (n + 31u) & ~31u;  // whole warps, so the ballots see full masks
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n_round; q += gridDim.x * blockDim.x) {
        bool go_on = false, to_shadow = false;
        uint32_t slot = 0;
        if (q < n) {
            slot = W.queue[cur][q];
            uint4 m = W.meta[slot];
            const uint4 hv = W.hit[slot];
            const float2 uv = W.huv[slot];
            const float4 o = W.ray_o[slot], d = W.ray_d[slot], tp = W.tp[slot], rd = W.rad[slot];
            Path path;
            path.o = mk(o.x, o.y, o.z);
            path.d = mk(d.x, d.y, d.z);
            path.tp = mk(tp.x, tp.y, tp.z);
            path.rad = mk(rd.x, rd.y, rd.z);
            path.bounce = int(m.z & 0xffu);
            path.sampled = (m.z & F_SAMPLED) != 0;
            Rng rng;
            const ulonglong2 r01 = W.rng[2 * slot], r23 = W.rng[2 * slot + 1];
            rng.s0 = r01.x;
            rng.s1 = r01.y;
            rng.s2 = r23.x;
            rng.s3 = r23.y;
            Sampler smp;
            smp.pixel_seed = m.w;
            smp.index = uint32_t(F.P.first_sample) + m.y;
            smp.set_bounce(path.bounce);
            ++rays;  // this bounce's ray (include/renderer.hpp:110)
            Hit h;
            h.kind = hv.x;
            h.index = hv.y;
            h.inst = hv.z;
            h.u = uv.x;
            h.v = uv.y;
            const bool hit = h.kind != PT_HIT_NONE;
            Rec rec;
            if (hit) fill(S, h, path.o, path.d, __uint_as_float(hv.w), rec);
            First first;
            if (AUX) {
                const float4 fa = W.first_albedo[slot], fn = W.first_normal[slot];
                first = {mk(fa.x, fa.y, fa.z), mk(fn.x, fn.y, fn.z)};
            }
            bool nee;
            Shadow sh;
            const int step = shade<AUX>(S, path, hit, rec, F.P.depth, smp, rng, first, nee, sh, rays);
            W.ray_o[slot] = make_float4(path.o.x, path.o.y, path.o.z, 0);
            W.ray_d[slot] = make_float4(path.d.x, path.d.y, path.d.z, 0);
            W.tp[slot] = make_float4(path.tp.x, path.tp.y, path.tp.z, 0);
            W.rad[slot] = make_float4(path.rad.x, path.rad.y, path.rad.z, 0);
            W.rng[2 * slot] = make_ulonglong2(rng.s0, rng.s1);
            W.rng[2 * slot + 1] = make_ulonglong2(rng.s2, rng.s3);
            if (AUX && path.bounce <= 1) {
                W.first_albedo[slot] = make_float4(first.albedo.x, first.albedo.y, first.albedo.z, 0);
                W.first_normal[slot] = make_float4(first.normal.x, first.normal.y, first.normal.z, 0);
            }
            uint32_t flags = (m.z & ~0x7ffu) | uint32_t(path.bounce) | F_IN_PATH | (path.sampled ? F_SAMPLED : 0u);
            if (nee) {
                W.sh_d[slot] = make_float4(sh.d.x, sh.d.y, sh.d.z, sh.t_max);
                W.sh_v[slot] = make_float4(sh.value.x, sh.value.y, sh.value.z, 0);
                to_shadow = true;
                if (step == STEP_DONE) flags |= F_DONE_PENDING;
                else go_on = true;
                m.z = flags;
                W.meta[slot] = m;
            } else if (step == STEP_DONE) {
                m.z = flags;
                W.meta[slot] = m;
                go_on = finish_sample<AUX>(F, W, slot);
            } else {
                m.z = flags;
                W.meta[slot] = m;
                go_on = true;
            }
        }
        push(W.shadow_q, &W.counts[2], to_shadow, slot);
        push(W.queue[nxt], &W.counts[nxt], go_on, slot);
    }
    if (rays_out) {
        unsigned long long total = rays;
        for (int off = 16; off > 0; off >>= 1) total += __shfl_down_sync(0xffffffffu, total, off);
        if ((threadIdx.x & 31) == 0 && total) atomicAdd(rays_out, total);
    }
}

// The occlusion test of each shadow ray.
template <bool AUX>
__global__ void __launch_bounds__(128) wf_shadow(PtSceneDev S, Frame F, WfView W, int cur) {
    PT_TRAV_STACK(stack, 128);
    const uint32_t n = W.counts[2];
    const int nxt = cur ^ 1;
    bool overflow = false;
    const uint32_t n_round = (n + 31u) & ~31u;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n_round; q += gridDim.x * blockDim.x) {
        bool go_on = false;
        uint32_t slot = 0;
        if (q < n) {
            slot = W.shadow_q[q];
            const float4 o = W.ray_o[slot], sd = W.sh_d[slot];
            Counts cnt;
            bool ovf = false;
            const bool blocked = occluded<false>(S, mk(o.x, o.y, o.z), mk(sd.x, sd.y, sd.z), 0.001f, sd.w, stack,
                                                 cnt, &ovf);
            overflow |= ovf;
            if (!blocked) {
                const float4 v = W.sh_v[slot];
                float4 r = W.rad[slot];
                r.x = r.x + v.x;
                r.y = r.y + v.y;
                r.z = r.z + v.z;
                W.rad[slot] = r;
            }
            uint4 m = W.meta[slot];
            if (m.z & F_DONE_PENDING) {
                m.z &= ~F_DONE_PENDING;
                W.meta[slot] = m;
                go_on = finish_sample<AUX>(F, W, slot);
            }
        }
        push(W.queue[nxt], &W.counts[nxt], go_on, slot);
    }
    if (overflow) atomicOr(S.status, PT_DEV_ERR_STACK);
}

}  // namespace

size_t pt_wavefront_bytes(uint32_t slots) {
    // 11 float4 + meta uint4 + 2 ulonglong2 + hit uint4 + float2 per slot, 3 queues, counters.
    return size_t(slots) * (11 * 16 + 16 + 32 + 16 + 8 + 3 * 4) + 4096;
}

namespace {

WfView carve(void* base, uint32_t slots) {
    char* p = static_cast<char*>(base);
    auto take = [&](size_t bytes) {
        char* r = p;
        p += (bytes + 255) & ~size_t(255);
        return r;
    };
    WfView W;
    W.slots = slots;
    W.ray_o = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.ray_d = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.tp = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.rad = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.acc = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.acc_albedo = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.acc_normal = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.first_albedo = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.first_normal = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.sh_d = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.sh_v = reinterpret_cast<float4*>(take(16 * size_t(slots)));
    W.meta = reinterpret_cast<uint4*>(take(16 * size_t(slots)));
    W.rng = reinterpret_cast<ulonglong2*>(take(32 * size_t(slots)));
    W.hit = reinterpret_cast<uint4*>(take(16 * size_t(slots)));
    W.huv = reinterpret_cast<float2*>(take(8 * size_t(slots)));
    W.queue[0] = reinterpret_cast<uint32_t*>(take(4 * size_t(slots)));
    W.queue[1] = reinterpret_cast<uint32_t*>(take(4 * size_t(slots)));
    W.shadow_q = reinterpret_cast<uint32_t*>(take(4 * size_t(slots)));
    W.counts = reinterpret_cast<uint32_t*>(take(256));
    return W;
}

int grid(uint32_t n, int threads, int sms, int per_sm) {
    const uint32_t want = (n + threads - 1) / threads;
    const uint32_t cap = uint32_t(sms * per_sm);
    return int(want < cap ? (want ? want : 1) : cap);
}

template <bool AUX>
cudaError_t run(const PtSceneDev& S, const PtRenderParams& p, void* scratch, uint32_t slots, int sms,
                cudaStream_t stream, uint32_t* host_counts) {
    Frame F;
    F.P = p;
    F.tiles_x = uint32_t((p.width + kTileW - 1) / kTileW);
    F.total_items = F.tiles_x * uint32_t((p.rows + kTileH - 1) / kTileH) * 32u;
    F.cam = {mk(p.cam.origin[0], p.cam.origin[1], p.cam.origin[2]), mk(p.cam.llc[0], p.cam.llc[1], p.cam.llc[2]),
             mk(p.cam.horizontal[0], p.cam.horizontal[1], p.cam.horizontal[2]),
             mk(p.cam.vertical[0], p.cam.vertical[1], p.cam.vertical[2])};
    WfView W = carve(scratch, slots);
    cudaError_t e = cudaMemsetAsync(W.counts, 0, 256, stream);
    if (e) return e;
    wf_init<AUX><<<grid(slots, 256, sms, 8), 256, 0, stream>>>(F, W);
    int cur = 0;
    // Waves until the ray queue drains. The queue length is read back every
    // few waves; waves launched on an empty queue do no work.
    for (int wave = 0;; ++wave) {
        for (int k = 0; k < 4; ++k) {
            wf_extend<<<sms * 8, 128, 0, stream>>>(S, W, cur);
            wf_shade<AUX><<<sms * 8, 128, 0, stream>>>(S, F, W, cur, p.rays);
            wf_shadow<AUX><<<sms * 8, 128, 0, stream>>>(S, F, W, cur);
            cur ^= 1;
        }
        if ((e = cudaGetLastError())) return e;
        if ((e = cudaMemcpyAsync(host_counts, W.counts + cur, 4, cudaMemcpyDeviceToHost, stream))) return e;
        if ((e = cudaStreamSynchronize(stream))) return e;
        if (*host_counts == 0) break;
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t pt_launch_wavefront(const PtSceneDev& S, const PtRenderParams& p, void* scratch, uint32_t slots,
                                int sms, cudaStream_t stream, uint32_t* host_counts) {
    return p.aux ? run<true>(S, p, scratch, slots, sms, stream, host_counts)
                 : run<false>(S, p, scratch, slots, sms, stream, host_counts);
}
