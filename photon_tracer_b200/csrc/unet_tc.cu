// Tensor-core 3x3 convolution for the U-Net (tcgen05, accumulators in TMEM).
//
// Implicit GEMM: M = a tile of 16 x 8 output pixels, N = Cout (16..256),
// K = 9 taps x Cin. Each K step is one tap and 32 input channels:
//   A: the 16 x 8 pixel box shifted by the tap, 32 channels, loaded by TMA
//      from the NHWC bf16 activations (out-of-image pixels read as zero,
//      which is the convolution's padding) -- 128 rows of 64 bytes;
//   B: the tap's weights for all Cout outputs and the same 32 channels, from
//      the [Cout][3][3][Cin] bf16 weights -- Cout rows of 64 bytes.
// Both land K-major with the 64-byte swizzle; two MMAs of K = 16 consume a
// step. One warp issues TMA, one thread issues MMAs, four warps drain the
// accumulator (bias, ReLU, bf16 or float) straight to global memory. CTAs
// are persistent over tiles with two TMEM accumulators.
//
// Every wait on an mbarrier is bounded (1 s); on expiry the kernel sets bit
// 0 of *status, lets the copies it issued land, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <algorithm>
#include <mutex>

#include "kernels.h"
#include "unet.h"

namespace {

constexpr int kTileX = 16, kTileY = 8, kM = kTileX * kTileY;  // 128 pixels = 128 TMEM lanes
constexpr int kKc = 32;                                        // input channels per K step (64 bytes)
constexpr int kStagesTile = 4;  // pipeline stages of the shifted-box form
constexpr int kThreads = 192;  // warp 0: TMA, warp 1: TMEM + MMA, warps 2-5: epilogue
constexpr int kMaxN = 256;     // output channels: two accumulators of N columns in 512
constexpr uint32_t kABytes = kM * kKc * 2;
constexpr unsigned long long kWaitNs = 1000000000ull;
// The halo form (Cout <= 64): an 8 x 16 pixel tile whose 10 x 18 halo box is
// loaded once per 32 input channels, as four planes of 8 channels (16 bytes
// per pixel) -- core matrices of 8 pixels x 8 channels -- so the A operand
// of each tap is the same buffer seen from the tap's offset.
constexpr int kHaloTX = 8, kHaloTY = 16, kHaloW = kHaloTX + 2, kHaloH = kHaloTY + 2;
constexpr uint32_t kPlane = kHaloW * kHaloH * 16;  // 2,880 bytes: one 8-channel plane
constexpr uint32_t kHaloBytes = 4 * kPlane;        // 11,520 bytes per 32 channels
constexpr uint32_t kHaloStage = 12288;             // rounded up to 1 KB

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of the given parity to complete; false after 1 s or
// when another role raised *abort.
__device__ bool wait_bar(uint32_t bar, uint32_t parity, const volatile int* abort) {
    if (try_wait(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    for (unsigned i = 1;; ++i) {
        if (try_wait(bar, parity)) return true;
        if ((i & 63) == 0) {
            if (abort && *abort) return false;
            if (now_ns() - t0 > kWaitNs) return false;
        }
    }
}

__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            int c4, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5, %6}], [%7];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
        : "memory");
}

// UMMA descriptor of a K-major operand without swizzle: core matrices of
// 8 rows x 16 bytes stored as 128 contiguous bytes, `lbo` bytes between the
// two core matrices of a K = 16 step, `sbo` bytes between 8-row groups.
__device__ __forceinline__ uint64_t plain_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3fff) | (uint64_t((lbo >> 4) & 0x3fff) << 16) |
           (uint64_t((sbo >> 4) & 0x3fff) << 32) | (uint64_t(1) << 46);
}

// UMMA shared-memory descriptor of a K-major operand with the 64-byte
// swizzle: rows of 64 bytes, 8-row groups 512 bytes apart (stride byte
// offset), leading byte offset unused (1), descriptor version 1.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t addr) {
    return uint64_t((addr >> 4) & 0x3fff) | (uint64_t(1) << 16) | (uint64_t(512 >> 4) << 32) | (uint64_t(1) << 46) |
           (uint64_t(4) << 61);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// The same load without the wait: several may be in flight before one
// tmem_wait(), and their registers are read only after it.
__device__ __forceinline__ void tmem_ld16_async(uint32_t addr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
}
__device__ __forceinline__ void tmem_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void bar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void pack_bf16(const float (&v)[16], uint4& a, uint4& b) {
    uint32_t w[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
        w[j] = *reinterpret_cast<const uint32_t*>(&h);
    }
    a = make_uint4(w[0], w[1], w[2], w[3]);
    b = make_uint4(w[4], w[5], w[6], w[7]);
}

struct TileGrid {
    int tiles_x, tiles_y, n, tx, ty;
    __device__ void origin(int t, int& x0, int& y0, int& b) const {
        x0 = (t % tiles_x) * tx;
        t /= tiles_x;
        y0 = (t % tiles_y) * ty;
        b = t / tiles_y;
    }
};

// Persistent: CTA c takes tiles c, c + gridDim.x, ... Two accumulators in
// TMEM (columns from 0 and from half the allocation, a power of two >= 2N)
// let the epilogue of one tile overlap the MMAs of the next; the TMA
// producer runs ahead across tile boundaries.
template <bool OUT_F32, bool HALO>
__global__ void __launch_bounds__(kThreads) conv_tc_kernel(const __grid_constant__ CUtensorMap tm_in,
                                                           const __grid_constant__ CUtensorMap tm_w, int B, int H,
                                                           int W, int Cin, int N, int tmem_cols, int stages,
                                                           int res, const float* __restrict__ bias, int relu,
                                                           const unet::ConvOut o, unsigned int* __restrict__ status) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int chunks = Cin / kKc, iters = HALO ? chunks : 9 * chunks;
    const uint32_t tap_bytes = uint32_t(N) * kKc * 2;  // one tap's weights for 32 channels
    // res (halo form only): all 9 x chunks weight boxes stay in shared memory
    // for the CTA's life, loaded once; the stages carry only the halo.
    const uint32_t w_bytes = res ? 9u * uint32_t(chunks) * tap_bytes : 0u;
    const uint32_t a_bytes = HALO ? kHaloStage : kABytes, b_bytes = res ? 0u : (HALO ? 9 * tap_bytes : tap_bytes);
    uint8_t* sw = smem;
    uint8_t* sa = smem + w_bytes;
    uint8_t* sb = sa + stages * a_bytes;
    // full[S], empty[S], acc_full[2], acc_empty[2], weights
    uint64_t* bars = reinterpret_cast<uint64_t*>(sb + stages * b_bytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * stages + 5);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + stages);
    const uint32_t acc_full0 = smem_u32(bars + 2 * stages), acc_empty0 = smem_u32(bars + 2 * stages + 2);
    const uint32_t wbar = smem_u32(bars + 2 * stages + 4);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    TileGrid grid;
    grid.tx = HALO ? kHaloTX : kTileX;
    grid.ty = HALO ? kHaloTY : kTileY;
    grid.tiles_x = (W + grid.tx - 1) / grid.tx;
    grid.tiles_y = (H + grid.ty - 1) / grid.ty;
    grid.n = grid.tiles_x * grid.tiles_y * B;

    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; ++s) {
            bar_init(full0 + 8 * s, 1);
            bar_init(empty0 + 8 * s, 1);
        }
        for (int a = 0; a < 2; ++a) {
            bar_init(acc_full0 + 8 * a, 1);
            bar_init(acc_empty0 + 8 * a, 4);  // one arrival per epilogue warp
        }
        bar_init(wbar, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // The bias once per CTA (zeros without one), read by the epilogue as
    // shared-memory broadcasts.
    __shared__ float sbias[kMaxN];
    for (int i = threadIdx.x; i < N; i += kThreads) sbias[i] = bias ? bias[i] : 0.0f;
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_in)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_w)) : "memory");
            if (res) {
                bar_expect_tx(wbar, w_bytes);
                for (int ch = 0; ch < chunks; ++ch)
                    for (int tap = 0; tap < 9; ++tap)
                        tma_load_3d(smem_u32(sw + (ch * 9 + tap) * tap_bytes), &tm_w, ch * kKc, tap, 0, wbar);
            }
            int g = 0;  // k steps issued so far, over all of this CTA's tiles
            for (int t = blockIdx.x; t < grid.n && ok; t += gridDim.x) {
                int x0, y0, b;
                grid.origin(t, x0, y0, b);
                for (int it = 0; it < iters; ++it, ++g) {
                    const int s = g % stages;
                    if (g >= stages && !wait_bar(empty0 + 8 * s, ((g / stages) - 1) & 1, abort)) {
                        ok = false;
                        break;
                    }
                    if (HALO) {
                        // the halo box of 32 channels (4 planes), and the 9 taps' weights for them
                        const int c0 = it * kKc;
                        bar_expect_tx(full0 + 8 * s, kHaloBytes + 9 * (res ? 0u : tap_bytes));
                        tma_load_5d(smem_u32(sa + s * a_bytes), &tm_in, 0, x0 - 1, y0 - 1, c0 / 8, b, full0 + 8 * s);
                        if (!res)
                            for (int tap = 0; tap < 9; ++tap)
                                tma_load_3d(smem_u32(sb + s * b_bytes + tap * tap_bytes), &tm_w, c0, tap, 0,
                                            full0 + 8 * s);
                    } else {
                        const int tap = it / chunks, c0 = (it - tap * chunks) * kKc;
                        bar_expect_tx(full0 + 8 * s, kABytes + b_bytes);
                        tma_load_4d(smem_u32(sa + s * a_bytes), &tm_in, c0, x0 + tap % 3 - 1, y0 + tap / 3 - 1, b,
                                    full0 + 8 * s);
                        tma_load_3d(smem_u32(sb + s * b_bytes), &tm_w, c0, tap, 0, full0 + 8 * s);
                    }
                }
            }
            // The copies issued into each stage have landed before the CTA can exit.
            for (int k = g > stages ? g - stages : 0; k < g; ++k)
                if (!wait_bar(full0 + 8 * (k % stages), (k / stages) & 1, nullptr)) ok = false;
            if (res && !wait_bar(wbar, 0, nullptr)) ok = false;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // kind::f16 instruction descriptor: f32 accumulate (bits 4-5 = 1),
            // A and B bf16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit
            // 17, M >> 4 at bit 24.
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(kM >> 4) << 24);
            int g = 0, i = 0;
            if (res && !wait_bar(wbar, 0, abort)) ok = false;
            for (int t = blockIdx.x; t < grid.n && ok; t += gridDim.x, ++i) {
                const int a = i & 1;
                if (i >= 2 && !wait_bar(acc_empty0 + 8 * a, ((i >> 1) - 1) & 1, abort)) {
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t d = tmem + uint32_t(a * (tmem_cols / 2));
                for (int it = 0; it < iters; ++it, ++g) {
                    const int s = g % stages;
                    if (!wait_bar(full0 + 8 * s, (g / stages) & 1, abort)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    if (HALO) {
                        // tap (dy, dx) reads the halo from offset (dy + 1, dx + 1): 8-pixel
                        // rows 10 pixels apart (SBO 160 B), K planes 2,880 B apart (LBO)
                        const uint32_t a0 = smem_u32(sa + s * a_bytes);
                        const uint32_t b0 = res ? smem_u32(sw + it * 9 * tap_bytes) : smem_u32(sb + s * b_bytes);
                        for (int tap = 0; tap < 9; ++tap) {
                            const uint32_t off = uint32_t((tap / 3) * kHaloW + tap % 3) * 16u;
                            const uint64_t bd = sw64_desc(b0 + tap * tap_bytes);
#pragma unroll
                            for (int k = 0; k < kKc / 16; ++k)
                                mma_bf16(d, plain_desc(a0 + 2 * k * kPlane + off, kPlane, kHaloW * 16),
                                         bd + uint64_t(2 * k), idesc, (it | tap | k) != 0);
                        }
                    } else {
                        const uint64_t ad = sw64_desc(smem_u32(sa + s * a_bytes));
                        const uint64_t bd = sw64_desc(smem_u32(sb + s * b_bytes));
#pragma unroll
                        for (int k = 0; k < kKc / 16; ++k)  // K = 16 per MMA: +32 bytes along the row
                            mma_bf16(d, ad + uint64_t(2 * k), bd + uint64_t(2 * k), idesc, (it | k) != 0);
                    }
                    mma_commit(empty0 + 8 * s);
                }
                mma_commit(acc_full0 + 8 * a);
            }
        }
    } else {
        const int q = warp & 3;  // the TMEM lane quarter this warp may read
        const int m = q * 32 + lane;
        int i = 0;
        for (int t = blockIdx.x; t < grid.n; t += gridDim.x, ++i) {
            const int a = i & 1;
            if (!__all_sync(0xffffffffu, wait_bar(acc_full0 + 8 * a, (i >> 1) & 1, abort))) {
                ok = false;
                break;
            }
            fence_after();
            int x0, y0, b;
            grid.origin(t, x0, y0, b);
            const int px = x0 + (m % grid.tx), py = y0 + (m / grid.tx);
            const bool valid = px < W && py < H;
            const size_t pix = (size_t(b) * H + (valid ? py : 0)) * W + (valid ? px : 0);
            // Pooling windows (x0, y0 even): the x neighbour is lane ^ 1, the
            // y neighbour lane ^ tx (a warp holds 32 / tx whole tile rows);
            // the even-x lane of the even row writes the window.
            const int ylane = HALO ? 8 : 16;
            const bool pool_writer = valid && !(lane & (1 | ylane));
            const size_t ppix = (size_t(b) * (H >> 1) + (py >> 1)) * (W >> 1) + (px >> 1);
            const uint32_t acc_addr = tmem + (uint32_t(q * 32) << 16) + uint32_t(a * (tmem_cols / 2));
            for (int c0 = 0; c0 < N; c0 += 32) {
              // two 16-column loads in flight per wait
              uint32_t r[2][16];
              tmem_ld16_async(acc_addr + uint32_t(c0), r[0]);
              if (c0 + 16 < N) tmem_ld16_async(acc_addr + uint32_t(c0 + 16), r[1]);
              tmem_wait();
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const int c = c0 + 16 * h;
                if (c >= N) break;
                float v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    v[j] = __uint_as_float(r[h][j]) + sbias[c + j];
                    if (relu) v[j] = fmaxf(v[j], 0.0f);
                }
                if (OUT_F32) {
                    if (!valid || !o.out) continue;
                    float4* dst = reinterpret_cast<float4*>(static_cast<float*>(o.out) + pix * o.stride + o.offset + c);
#pragma unroll
                    for (int j = 0; j < 4; ++j) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
                    continue;
                }
                uint4 w0, w1;
                pack_bf16(v, w0, w1);
                if (valid && o.out) {
                    uint4* dst = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(o.out) + pix * o.stride + o.offset + c);
                    dst[0] = w0;
                    dst[1] = w1;
                }
                if (valid && o.out2) {
                    if (o.up2) {
                        // nearest 2x: the four pixels (2px + i, 2py + j) of the finer level
#pragma unroll
                        for (int j = 0; j < 2; ++j)
#pragma unroll
                            for (int i = 0; i < 2; ++i) {
                                const size_t q2 = (size_t(b) * 2 * H + 2 * py + j) * (2 * W) + 2 * px + i;
                                uint4* dst = reinterpret_cast<uint4*>(o.out2 + q2 * o.stride2 + o.offset2 + c);
                                dst[0] = w0;
                                dst[1] = w1;
                            }
                    } else {
                        uint4* dst = reinterpret_cast<uint4*>(o.out2 + pix * o.stride2 + o.offset2 + c);
                        dst[0] = w0;
                        dst[1] = w1;
                    }
                }
                if (o.pool) {
                    // max commutes with the monotonic bf16 rounding: pooling the
                    // floats then rounding equals pooling the stored bf16 values.
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        v[j] = fmaxf(v[j], __shfl_xor_sync(0xffffffffu, v[j], 1));
                        v[j] = fmaxf(v[j], __shfl_xor_sync(0xffffffffu, v[j], ylane));
                    }
                    if (pool_writer) {
                        uint4 p0, p1;
                        pack_bf16(v, p0, p1);
                        uint4* dst = reinterpret_cast<uint4*>(o.pool + ppix * N + c);
                        dst[0] = p0;
                        dst[1] = p1;
                    }
                }
              }
            }
            // This warp's reads of the accumulator are done: the MMA warp may reuse it.
            fence_before();
            __syncwarp();
            if (lane == 0) bar_arrive(acc_empty0 + 8 * a);
        }
    }

    if (!ok) {
        *abort = 1;
        atomicOr(status, 1u);
    }
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Pipeline stages and dynamic shared memory of the two forms.
#ifndef PT_CONV_HALO_MAX_N
#define PT_CONV_HALO_MAX_N 64
#endif
// The halo form's A descriptors (LBO = one 2,880-byte plane, SBO = one
// 160-byte halo row) reach at most 15 * 160 + 7 * 16 + 2,880 + 16 bytes past
// a start of at most 2 * 2,880 + (2 * 10 + 2) * 16: exactly the 11,520 bytes
// of the stage's halo.
size_t conv_smem(bool halo, bool res, int Cin, int N, int stages) {
    const size_t tap = size_t(N) * kKc * 2;
    const size_t w = res ? 9 * tap * size_t(Cin / kKc) : 0;
    const size_t a = halo ? kHaloStage : kABytes, b = res ? 0 : (halo ? 9 : 1) * tap;
    return 1024 + w + stages * (a + b) + (2 * stages + 5) * 8 + 8;
}

// Shared memory layout of one launch. The halo form keeps its weights
// resident when they take at most 80 KB, with as many halo stages (2 to 6)
// as leave three CTAs per SM, else two (228 KB per SM, 1 KB reserved and
// 1 KB of bias per CTA); bigger weights stream with each stage.
struct ConvPlan {
    bool halo, res;
    int stages;
    size_t smem;
};
constexpr size_t kSmemPerSM = 228 * 1024, kResMaxBytes = 80 * 1024;
#ifndef PT_CONV_RESIDENT
#define PT_CONV_RESIDENT 1
#endif
ConvPlan conv_plan(bool halo, int Cin, int N) {
    ConvPlan p{halo, false, halo ? (N <= 32 ? 3 : 2) : kStagesTile, 0};
    if (PT_CONV_RESIDENT && halo && size_t(9) * Cin * N * 2 <= kResMaxBytes) {
        for (int ctas = 3; ctas >= 2 && !p.res; --ctas)
            for (int st = 6; st >= 2; --st)
                if (conv_smem(true, true, Cin, N, st) <= kSmemPerSM / ctas - 2048) {
                    p.res = true;
                    p.stages = st;
                    break;
                }
    }
    p.smem = conv_smem(halo, p.res, Cin, N, p.stages);
    return p;
}

// CTAs that fit on all SMs at once: the kernel's resident blocks per SM
// (shared memory, threads, registers), capped by the TMEM columns each holds.
int grid_size(int cols, size_t smem, const void* fn) {
    static int sms[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!sms[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        sms[dev] = n > 0 ? n : 1;
    }
    const int per_sm = std::min(pt_resident_blocks(fn, kThreads, smem), 512 / cols);
    return sms[dev] * std::max(per_sm, 1);
}

// ---- weight gradient -------------------------------------------------------
// dW[co][tap][ci] = sum over pixels p of dY[p][co] * X[p + offset(tap)][ci]:
// per tap a GEMM with M = Cout (padded to 128), N = Cin (padded to a
// multiple of 64), K = pixels. A K step is a 16 x 4 pixel box: dY unshifted
// and X shifted by the tap (zeros outside the image), both channel-contiguous
// -- MN-major operands, 128-byte swizzle, one 64-channel TMA box per 64
// rows of M or N. A CTA reduces one tap over a range of pixel boxes in TMEM
// and adds its partial sums to dW with float atomics.
constexpr int kWgBoxX = 16, kWgBoxY = 4, kWgK = kWgBoxX * kWgBoxY;  // 64 pixels per K step
constexpr int kWgStages = 4;
constexpr uint32_t kWgBox = kWgK * 64 * 2;  // one 64-channel box: 8 KB

// UMMA descriptor of an MN-major operand with the 128-byte swizzle: 64
// elements of M or N per 128-byte row, one row per K index; 8-row groups
// 1024 bytes apart (stride byte offset), 64-element blocks of M or N one
// 8 KB box apart (leading byte offset), descriptor version 1.
__device__ __forceinline__ uint64_t mn_sw128_desc(uint32_t addr) {
    return uint64_t((addr >> 4) & 0x3fff) | (uint64_t(kWgBox >> 4) << 16) | (uint64_t(1024 >> 4) << 32) |
           (uint64_t(1) << 46) | (uint64_t(2) << 61);
}

__global__ void __launch_bounds__(kThreads) wgrad_tc_kernel(const __grid_constant__ CUtensorMap tm_dy,
                                                            const __grid_constant__ CUtensorMap tm_x, int B, int H,
                                                            int W, int Cin, int Cout, int N, int tmem_cols, int splits,
                                                            float* __restrict__ dw, unsigned int* __restrict__ status) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int nb = N / 64;  // X boxes per stage
    const uint32_t stage_bytes = (2 + nb) * kWgBox;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kWgStages * stage_bytes);  // full[S], empty[S], done
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kWgStages + 1);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kWgStages), done = smem_u32(bars + 2 * kWgStages);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tap = blockIdx.x % 9, split = blockIdx.x / 9;
    const int bx = (W + kWgBoxX - 1) / kWgBoxX, by = (H + kWgBoxY - 1) / kWgBoxY;
    const long boxes = long(bx) * by * B;
    const long k0 = boxes * split / splits, k1 = boxes * (split + 1) / splits;
    const int iters = int(k1 - k0);
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kWgStages; ++s) {
            bar_init(full0 + 8 * s, 1);
            bar_init(empty0 + 8 * s, 1);
        }
        bar_init(done, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_dy)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_x)) : "memory");
            int it = 0;
            for (; it < iters; ++it) {
                const int s = it % kWgStages;
                if (it >= kWgStages && !wait_bar(empty0 + 8 * s, ((it / kWgStages) - 1) & 1, abort)) {
                    ok = false;
                    break;
                }
                long k = k0 + it;
                const int x0 = int(k % bx) * kWgBoxX;
                k /= bx;
                const int y0 = int(k % by) * kWgBoxY, b = int(k / by);
                const uint32_t st = smem_u32(smem + s * stage_bytes), bar = full0 + 8 * s;
                bar_expect_tx(bar, stage_bytes);
                tma_load_4d(st, &tm_dy, 0, x0, y0, b, bar);
                tma_load_4d(st + kWgBox, &tm_dy, 64, x0, y0, b, bar);
                for (int j = 0; j < nb; ++j) tma_load_4d(st + (2 + j) * kWgBox, &tm_x, 64 * j, x0 + dx, y0 + dy, b, bar);
            }
            for (int k = it > kWgStages ? it - kWgStages : 0; k < it; ++k)
                if (!wait_bar(full0 + 8 * (k % kWgStages), (k / kWgStages) & 1, nullptr)) ok = false;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // kind::f16: f32 accumulate, A and B bf16, both MN-major (bits 15,
            // 16), N >> 3 at bit 17, M = 128 >> 4 at bit 24.
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                                   (uint32_t(N >> 3) << 17) | (uint32_t(128 >> 4) << 24);
            for (int it = 0; it < iters; ++it) {
                const int s = it % kWgStages;
                if (!wait_bar(full0 + 8 * s, (it / kWgStages) & 1, abort)) {
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t st = smem_u32(smem + s * stage_bytes);
                const uint64_t ad = mn_sw128_desc(st), bd = mn_sw128_desc(st + 2 * kWgBox);
#pragma unroll
                for (int k = 0; k < kWgK / 16; ++k)  // K = 16 rows = two 1024-byte groups per MMA
                    mma_bf16(tmem, ad + uint64_t(k * (2048 >> 4)), bd + uint64_t(k * (2048 >> 4)), idesc,
                             (it | k) != 0);
                mma_commit(empty0 + 8 * s);
            }
            mma_commit(done);
        }
    } else {
        const int q = warp & 3;
        const int co = q * 32 + lane;
        if (iters > 0 && __all_sync(0xffffffffu, wait_bar(done, 0, abort))) {
            fence_after();
            for (int c = 0; c < N; c += 16) {
                float v[16];
                tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(c), v);
                if (co >= Cout) continue;
                float* dst = dw + (size_t(co) * 9 + tap) * Cin + c;
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (c + j < Cin) atomicAdd(dst + j, v[j]);
            }
        } else if (iters > 0) {
            ok = false;
        }
    }

    if (!ok) {
        *abort = 1;
        atomicOr(status, 1u);
    }
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
    }
}

}  // namespace

namespace unet {

cudaError_t conv_fwd_tc(const ConvShape& s, const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias,
                        bool relu, const ConvOut& o, bool out_f32, unsigned int* status, cudaStream_t st) {
    const int N = s.Cout;
    const int esz = out_f32 ? 4 : 2;
    if (s.Cin % kKc || N % 16 || N < 16 || N > 256 || s.B < 1 || s.H < 1 || s.W < 1) return cudaErrorNotSupported;
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(w)) % 16) return cudaErrorNotSupported;
    if (reinterpret_cast<uintptr_t>(o.out) % 16 || (size_t(o.offset) * esz) % 16 || (size_t(o.stride) * esz) % 16)
        return cudaErrorNotSupported;
    if (out_f32 && (o.out2 || o.pool)) return cudaErrorNotSupported;
    if (reinterpret_cast<uintptr_t>(o.out2) % 16 || (size_t(o.offset2) * 2) % 16 || (size_t(o.stride2) * 2) % 16)
        return cudaErrorNotSupported;
    if (o.pool && (reinterpret_cast<uintptr_t>(o.pool) % 16 || s.H % 2 || s.W % 2)) return cudaErrorNotSupported;
    PFN_cuTensorMapEncodeTiled_v12000 encode = encode_fn();
    if (!encode) return cudaErrorNotSupported;

    // The halo form for Cout <= 64 (where re-reading the shifted box per tap
    // bounds the kernel), the shifted-box form otherwise or if the halo's
    // tensor map is refused.
    bool halo = N <= PT_CONV_HALO_MAX_N;
    CUtensorMap tm_in, tm_w;
    if (halo) {
        // [B][H][W][Cin] seen as (8 channels, x, y, channel group, image): the
        // box (8, 10, 18, 4, 1) lands as four 8-channel planes of the halo.
        const cuuint64_t dims[5] = {8, cuuint64_t(s.W), cuuint64_t(s.H), cuuint64_t(s.Cin / 8), cuuint64_t(s.B)};
        const cuuint64_t strides[4] = {cuuint64_t(s.Cin) * 2, cuuint64_t(s.W) * s.Cin * 2, 16,
                                       cuuint64_t(s.H) * s.W * s.Cin * 2};
        const cuuint32_t box[5] = {8, kHaloW, kHaloH, 4, 1};
        const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
        halo = encode(&tm_in, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(in), dims, strides, box,
                      estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    if (!halo) {
        const cuuint64_t dims[4] = {cuuint64_t(s.Cin), cuuint64_t(s.W), cuuint64_t(s.H), cuuint64_t(s.B)};
        const cuuint64_t strides[3] = {cuuint64_t(s.Cin) * 2, cuuint64_t(s.W) * s.Cin * 2,
                                       cuuint64_t(s.H) * s.W * s.Cin * 2};
        const cuuint32_t box[4] = {kKc, kTileX, kTileY, 1};
        const cuuint32_t estr[4] = {1, 1, 1, 1};
        if (encode(&tm_in, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(in), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorNotSupported;
    }
    {
        const cuuint64_t dims[3] = {cuuint64_t(s.Cin), 9, cuuint64_t(N)};
        const cuuint64_t strides[2] = {cuuint64_t(s.Cin) * 2, cuuint64_t(9) * s.Cin * 2};
        const cuuint32_t box[3] = {kKc, 1, cuuint32_t(N)};
        const cuuint32_t estr[3] = {1, 1, 1};
        if (encode(&tm_w, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(w), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorNotSupported;
    }
    int cols = 32;
    while (cols < 2 * N) cols *= 2;  // two accumulators
    const ConvPlan plan = conv_plan(halo, s.Cin, N);
    const size_t smem = plan.smem;
    const int stages = plan.stages;
    const int tx = halo ? kHaloTX : kTileX, ty = halo ? kHaloTY : kTileY;
    const long tiles = long((s.W + tx - 1) / tx) * ((s.H + ty - 1) / ty) * s.B;
    if (tiles > 0x7fffffffL) return cudaErrorNotSupported;
    const void* fn = out_f32 ? (halo ? reinterpret_cast<const void*>(conv_tc_kernel<true, true>)
                                     : reinterpret_cast<const void*>(conv_tc_kernel<true, false>))
                             : (halo ? reinterpret_cast<const void*>(conv_tc_kernel<false, true>)
                                     : reinterpret_cast<const void*>(conv_tc_kernel<false, false>));
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e) return e;
    const long g = grid_size(cols, smem, fn);
    const unsigned blocks = unsigned(tiles < g ? tiles : g);
#define PT_CONV_LAUNCH(F32, HALO)                                                                                     \
    conv_tc_kernel<F32, HALO><<<blocks, kThreads, smem, st>>>(tm_in, tm_w, s.B, s.H, s.W, s.Cin, N, cols, stages,       \
                                                             plan.res ? 1 : 0, bias, relu, o, status)
    if (out_f32) {
        if (halo)
            PT_CONV_LAUNCH(true, true);
        else
            PT_CONV_LAUNCH(true, false);
    } else {
        if (halo)
            PT_CONV_LAUNCH(false, true);
        else
            PT_CONV_LAUNCH(false, false);
    }
#undef PT_CONV_LAUNCH
    return cudaGetLastError();
}

cudaError_t conv_wgrad_tc(const ConvShape& s, const __nv_bfloat16* in, const __nv_bfloat16* dout, float* dw,
                          unsigned int* status, cudaStream_t st) {
    const int N = (s.Cin + 63) / 64 * 64;
    if (s.Cout > 128 || s.Cout % 8 || s.Cin % 8 || N > 256 || s.B < 1 || s.H < 1 || s.W < 1)
        return cudaErrorNotSupported;
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(dout)) % 16) return cudaErrorNotSupported;
    PFN_cuTensorMapEncodeTiled_v12000 encode = encode_fn();
    if (!encode) return cudaErrorNotSupported;
    CUtensorMap tm_dy, tm_x;
    const cuuint32_t box[4] = {64, kWgBoxX, kWgBoxY, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    {
        const cuuint64_t dims[4] = {cuuint64_t(s.Cout), cuuint64_t(s.W), cuuint64_t(s.H), cuuint64_t(s.B)};
        const cuuint64_t strides[3] = {cuuint64_t(s.Cout) * 2, cuuint64_t(s.W) * s.Cout * 2,
                                       cuuint64_t(s.H) * s.W * s.Cout * 2};
        if (encode(&tm_dy, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(dout), dims, strides, box,
                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorNotSupported;
    }
    {
        const cuuint64_t dims[4] = {cuuint64_t(s.Cin), cuuint64_t(s.W), cuuint64_t(s.H), cuuint64_t(s.B)};
        const cuuint64_t strides[3] = {cuuint64_t(s.Cin) * 2, cuuint64_t(s.W) * s.Cin * 2,
                                       cuuint64_t(s.H) * s.W * s.Cin * 2};
        if (encode(&tm_x, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(in), dims, strides, box,
                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorNotSupported;
    }
    int cols = 32;
    while (cols < N) cols *= 2;
    const size_t smem = 1024 + kWgStages * size_t(2 + N / 64) * kWgBox + (2 * kWgStages + 1) * 8 + 8;
    cudaError_t e = cudaFuncSetAttribute(wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e) return e;
    const long boxes = long((s.W + kWgBoxX - 1) / kWgBoxX) * ((s.H + kWgBoxY - 1) / kWgBoxY) * s.B;
    // About two CTAs per SM over the 9 taps, at least 8 boxes each.
    const int target = grid_size(cols, smem, reinterpret_cast<const void*>(wgrad_tc_kernel));
    long splits = (2L * target + 8) / 9;
    if (splits > boxes / 8) splits = boxes / 8;
    if (splits < 1) splits = 1;
    wgrad_tc_kernel<<<unsigned(9 * splits), kThreads, smem, st>>>(tm_dy, tm_x, s.B, s.H, s.W, s.Cin, s.Cout, N, cols,
                                                                 int(splits), dw, status);
    return cudaGetLastError();
}

}  // namespace unet
