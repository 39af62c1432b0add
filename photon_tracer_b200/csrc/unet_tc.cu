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
// accumulator (bias, ReLU, bf16 or float) straight to global memory.
//
// Every wait on an mbarrier is bounded (1 s); on expiry the kernel sets bit
// 0 of *status, lets the copies it issued land, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "unet.h"

namespace {

constexpr int kTileX = 16, kTileY = 8, kM = kTileX * kTileY;  // 128 pixels = 128 TMEM lanes
constexpr int kKc = 32;                                        // input channels per K step (64 bytes)
constexpr int kStages = 4;
constexpr int kThreads = 192;  // warp 0: TMA, warp 1: TMEM + MMA, warps 2-5: epilogue
constexpr uint32_t kABytes = kM * kKc * 2;
constexpr unsigned long long kWaitNs = 1000000000ull;

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

template <bool OUT_F32>
__global__ void __launch_bounds__(kThreads) conv_tc_kernel(const __grid_constant__ CUtensorMap tm_in,
                                                           const __grid_constant__ CUtensorMap tm_w, int H, int W,
                                                           int Cin, int N, int tmem_cols,
                                                           const float* __restrict__ bias, int relu,
                                                           void* __restrict__ out, int out_stride, int out_offset,
                                                           unsigned int* __restrict__ status) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t b_bytes = uint32_t(N) * kKc * 2;
    uint8_t* sa = smem;
    uint8_t* sb = smem + kStages * kABytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sb + kStages * b_bytes);  // full[S], empty[S], done
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 1);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages), done = smem_u32(bars + 2 * kStages);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_x = (W + kTileX - 1) / kTileX, tiles_y = (H + kTileY - 1) / kTileY;
    int t = blockIdx.x;
    const int x0 = (t % tiles_x) * kTileX;
    t /= tiles_x;
    const int y0 = (t % tiles_y) * kTileY;
    const int b = t / tiles_y;
    const int chunks = Cin / kKc, iters = 9 * chunks;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
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
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_in)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_w)) : "memory");
            int it = 0;
            for (; it < iters; ++it) {
                const int s = it % kStages;
                if (it >= kStages && !wait_bar(empty0 + 8 * s, ((it / kStages) - 1) & 1, abort)) {
                    ok = false;
                    break;
                }
                const int tap = it / chunks, c0 = (it - tap * chunks) * kKc;
                bar_expect_tx(full0 + 8 * s, kABytes + b_bytes);
                tma_load_4d(smem_u32(sa + s * kABytes), &tm_in, c0, x0 + tap % 3 - 1, y0 + tap / 3 - 1, b, full0 + 8 * s);
                tma_load_3d(smem_u32(sb + s * b_bytes), &tm_w, c0, tap, 0, full0 + 8 * s);
            }
            // The copies issued into each stage have landed before the CTA can exit.
            for (int k = it > kStages ? it - kStages : 0; k < it; ++k)
                if (!wait_bar(full0 + 8 * (k % kStages), (k / kStages) & 1, nullptr)) ok = false;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // kind::f16 instruction descriptor: f32 accumulate (bits 4-5 = 1),
            // A and B bf16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit
            // 17, M >> 4 at bit 24.
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(kM >> 4) << 24);
            for (int it = 0; it < iters; ++it) {
                const int s = it % kStages;
                if (!wait_bar(full0 + 8 * s, (it / kStages) & 1, abort)) {
                    ok = false;
                    break;
                }
                fence_after();
                const uint64_t ad = sw64_desc(smem_u32(sa + s * kABytes)), bd = sw64_desc(smem_u32(sb + s * b_bytes));
#pragma unroll
                for (int k = 0; k < kKc / 16; ++k)  // K = 16 per MMA: +32 bytes along the row
                    mma_bf16(tmem, ad + uint64_t(2 * k), bd + uint64_t(2 * k), idesc, (it | k) != 0);
                mma_commit(empty0 + 8 * s);
            }
            mma_commit(done);
        }
    } else {
        const int q = warp & 3;  // the TMEM lane quarter this warp may read
        const int m = q * 32 + lane;
        const int px = x0 + (m % kTileX), py = y0 + (m / kTileX);
        const bool valid = px < W && py < H;
        const bool got = __all_sync(0xffffffffu, wait_bar(done, 0, abort));
        if (got) {
            fence_after();
            const size_t pix = (size_t(b) * H + (valid ? py : 0)) * W + (valid ? px : 0);
            for (int c = 0; c < N; c += 16) {
                float v[16];
                tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(c), v);
                if (!valid) continue;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    v[i] += bias ? bias[c + i] : 0.0f;
                    if (relu) v[i] = fmaxf(v[i], 0.0f);
                }
                if (OUT_F32) {
                    float4* dst = reinterpret_cast<float4*>(static_cast<float*>(out) + pix * out_stride + out_offset + c);
#pragma unroll
                    for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                } else {
                    uint32_t w[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                        w[i] = *reinterpret_cast<const uint32_t*>(&h);
                    }
                    uint4* dst = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(out) + pix * out_stride + out_offset + c);
                    dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
                    dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
                }
            }
        } else {
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

size_t smem_bytes(int N) { return 1024 + kStages * (kABytes + size_t(N) * kKc * 2) + (2 * kStages + 1) * 8 + 8; }

}  // namespace

namespace unet {

cudaError_t conv_fwd_tc(const ConvShape& s, const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias,
                        bool relu, void* out, bool out_f32, int out_stride, int out_offset, unsigned int* status,
                        cudaStream_t st) {
    const int N = s.Cout;
    const int esz = out_f32 ? 4 : 2;
    if (s.Cin % kKc || N % 16 || N < 16 || N > 256 || s.B < 1 || s.H < 1 || s.W < 1) return cudaErrorNotSupported;
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(w)) % 16) return cudaErrorNotSupported;
    if (reinterpret_cast<uintptr_t>(out) % 16 || (size_t(out_offset) * esz) % 16 || (size_t(out_stride) * esz) % 16)
        return cudaErrorNotSupported;
    PFN_cuTensorMapEncodeTiled_v12000 encode = encode_fn();
    if (!encode) return cudaErrorNotSupported;

    CUtensorMap tm_in, tm_w;
    {
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
    while (cols < N) cols *= 2;
    const size_t smem = smem_bytes(N);
    const long tiles = long((s.W + kTileX - 1) / kTileX) * ((s.H + kTileY - 1) / kTileY) * s.B;
    if (tiles > 0x7fffffffL) return cudaErrorNotSupported;
    cudaError_t e;
    if (out_f32) {
        e = cudaFuncSetAttribute(conv_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e) return e;
        conv_tc_kernel<true><<<unsigned(tiles), kThreads, smem, st>>>(tm_in, tm_w, s.H, s.W, s.Cin, N, cols, bias, relu,
                                                                      out, out_stride, out_offset, status);
    } else {
        e = cudaFuncSetAttribute(conv_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e) return e;
        conv_tc_kernel<false><<<unsigned(tiles), kThreads, smem, st>>>(tm_in, tm_w, s.H, s.W, s.Cin, N, cols, bias,
                                                                       relu, out, out_stride, out_offset, status);
    }
    return cudaGetLastError();
}

}  // namespace unet
