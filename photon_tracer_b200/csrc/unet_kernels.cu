// Building blocks of the U-Net denoiser: 3x3 convolutions (forward, and the
// two halves of backward), 2x2 max pooling, nearest 2x upsampling, channel
// concatenation, the input/output transforms, L1 loss on log radiance, and
// Adam. Activations are NHWC bfloat16 with the channel count padded to a
// multiple of 32; gradients of activations are float; weights are
// [Cout][3][3][Cin] (the K-major operand layout of an implicit GEMM).
//
// These are the CUDA-core kernels; the tensor-core forward (unet_tc.cu)
// replaces conv_fwd where the shapes allow and is checked against it.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "unet.h"

namespace {

template <class T>
__device__ __forceinline__ float to_f(T x);
template <>
__device__ __forceinline__ float to_f<float>(float x) { return x; }
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }

template <class T>
__device__ __forceinline__ T from_f(float x);
template <>
__device__ __forceinline__ float from_f<float>(float x) { return x; }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }

constexpr int kCoTile = 16;

// out[b,y,x,co] = act(bias[co] + sum_{dy,dx,ci} in[b,y+dy-1,x+dx-1,ci] * w[co][dy][dx][ci])
// One thread: one pixel, 16 output channels. The block stages one tap's
// weights for its 16 output channels in shared memory.
template <class TI, class TO>
__global__ void __launch_bounds__(128) conv_fwd_kernel(int B, int H, int W, int Cin, int Cout,
                                                       const TI* __restrict__ in, const __nv_bfloat16* __restrict__ w,
                                                       const float* __restrict__ bias, int relu, TO* __restrict__ out,
                                                       int out_stride, int out_offset) {
    extern __shared__ float ws[];  // kCoTile x Cin
    const int co0 = blockIdx.y * kCoTile;
    const long p = long(blockIdx.x) * blockDim.x + threadIdx.x;
    const long P = long(B) * H * W;
    const bool active = p < P;
    int b = 0, y = 0, x = 0;
    if (active) {
        b = int(p / (long(H) * W));
        const int r = int(p - long(b) * H * W);
        y = r / W;
        x = r - y * W;
    }
    float acc[kCoTile];
#pragma unroll
    for (int j = 0; j < kCoTile; ++j) acc[j] = (bias && co0 + j < Cout) ? bias[co0 + j] : 0.0f;
    for (int tap = 0; tap < 9; ++tap) {
        __syncthreads();
        for (int i = threadIdx.x; i < kCoTile * Cin; i += blockDim.x) {
            const int j = i / Cin, ci = i - j * Cin;
            ws[i] = co0 + j < Cout ? __bfloat162float(w[(size_t(co0 + j) * 9 + tap) * Cin + ci]) : 0.0f;
        }
        __syncthreads();
        if (!active) continue;
        const int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
        if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
        const TI* src = in + ((size_t(b) * H + yy) * W + xx) * Cin;
        for (int ci = 0; ci < Cin; ++ci) {
            const float v = to_f(src[ci]);
#pragma unroll
            for (int j = 0; j < kCoTile; ++j) acc[j] += v * ws[j * Cin + ci];
        }
    }
    if (!active) return;
    TO* dst = out + size_t(p) * out_stride + out_offset;
#pragma unroll
    for (int j = 0; j < kCoTile; ++j)
        if (co0 + j < Cout) dst[co0 + j] = from_f<TO>(relu ? fmaxf(acc[j], 0.0f) : acc[j]);
}

// dw[co][tap][ci] += sum_p dout[p][co] * in[p + tap][ci]; db[co] += sum_p dout[p][co].
// Block: one tap, 16 output channels, 32 input channels, a range of pixels.
__global__ void __launch_bounds__(256) conv_wgrad_kernel(int B, int H, int W, int Cin, int Cout,
                                                         const __nv_bfloat16* __restrict__ in,
                                                         const float* __restrict__ dout, float* __restrict__ dw,
                                                         float* __restrict__ db, long px_per_block) {
    __shared__ float so[64][kCoTile];
    __shared__ float si[64][33];
    const int tap = blockIdx.x % 9;
    const int ci0 = (blockIdx.x / 9) * 32;
    const int co0 = blockIdx.y * kCoTile;
    const long P = long(B) * H * W;
    const long p_begin = long(blockIdx.z) * px_per_block;
    const long p_end = p_begin + px_per_block < P ? p_begin + px_per_block : P;
    const int t = threadIdx.x;
    const int pj = t / 32, pci = t % 32;  // this thread's (co pair, ci)
    float acc0 = 0, acc1 = 0, bacc = 0;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    for (long p0 = p_begin; p0 < p_end; p0 += 64) {
        __syncthreads();
        for (int i = t; i < 64 * kCoTile; i += 256) {
            const int r = i / kCoTile, j = i % kCoTile;
            const long p = p0 + r;
            so[r][j] = (p < p_end && co0 + j < Cout) ? dout[size_t(p) * Cout + co0 + j] : 0.0f;
        }
        for (int i = t; i < 64 * 32; i += 256) {
            const int r = i / 32, c = i % 32;
            const long p = p0 + r;
            float v = 0;
            if (p < p_end && ci0 + c < Cin) {
                const int b = int(p / (long(H) * W));
                const int rr = int(p - long(b) * H * W);
                const int y = rr / W + dy, x = rr % W + dx;
                if (y >= 0 && y < H && x >= 0 && x < W) v = __bfloat162float(in[((size_t(b) * H + y) * W + x) * Cin + ci0 + c]);
            }
            si[r][c] = v;
        }
        __syncthreads();
#pragma unroll 8
        for (int r = 0; r < 64; ++r) {
            const float v = si[r][pci];
            acc0 += so[r][2 * pj] * v;
            acc1 += so[r][2 * pj + 1] * v;
        }
        if (tap == 0 && ci0 == 0 && t < kCoTile)
            for (int r = 0; r < 64; ++r) bacc += so[r][t];
    }
    const int ci = ci0 + pci;
    if (ci < Cin) {
        if (co0 + 2 * pj < Cout) atomicAdd(&dw[(size_t(co0 + 2 * pj) * 9 + tap) * Cin + ci], acc0);
        if (co0 + 2 * pj + 1 < Cout) atomicAdd(&dw[(size_t(co0 + 2 * pj + 1) * 9 + tap) * Cin + ci], acc1);
    }
    if (db && tap == 0 && ci0 == 0 && t < kCoTile && co0 + t < Cout) atomicAdd(&db[co0 + t], bacc);
}

// db[c] += sum over pixels of g[p][c] (C <= 256): R = 256 / C rows of
// threads per block stride over the block's pixels, then one row sums.
__global__ void __launch_bounds__(256) bias_grad_kernel(long pixels, int C, const float* __restrict__ g,
                                                        float* __restrict__ db, long px_per_block) {
    __shared__ float part[256];
    const int R = 256 / C;
    const int t = threadIdx.x, c = t % C, r = t / C;
    const long p0 = long(blockIdx.x) * px_per_block;
    const long p1 = p0 + px_per_block < pixels ? p0 + px_per_block : pixels;
    float acc = 0.0f;
    if (r < R)
        for (long p = p0 + r; p < p1; p += R) acc += g[p * C + c];
    part[t] = acc;
    __syncthreads();
    if (r == 0) {
        for (int k = 1; k < R; ++k) acc += part[k * C + c];
        atomicAdd(db + c, acc);
    }
}

// w_t[ci][tap][co] = w[co][8 - tap][ci]: the weights of the transposed
// convolution that carries gradients back to a layer's input.
__global__ void flip_transpose_kernel(int Cin, int Cout, const __nv_bfloat16* __restrict__ w,
                                      __nv_bfloat16* __restrict__ wt) {
    const long n = long(Cin) * 9 * Cout;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int co = int(i % Cout);
        const int tap = int((i / Cout) % 9);
        const int ci = int(i / (long(Cout) * 9));
        wt[i] = w[(size_t(co) * 9 + (8 - tap)) * Cin + ci];
    }
}

// Gradient through ReLU: g *= (y > 0), converted to bf16 for the next conv.
__global__ void relu_grad_kernel(long n, const __nv_bfloat16* __restrict__ y, float* __restrict__ g,
                                 __nv_bfloat16* __restrict__ g16) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const float v = __bfloat162float(y[i]) > 0.0f ? g[i] : 0.0f;
        g[i] = v;
        if (g16) g16[i] = __float2bfloat16_rn(v);
    }
}

__global__ void to_bf16_kernel(long n, const float* __restrict__ g, __nv_bfloat16* __restrict__ g16) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        g16[i] = __float2bfloat16_rn(g[i]);
}

// 2x2 max pooling (H, W even).
__global__ void pool_fwd_kernel(int B, int H, int W, int C, const __nv_bfloat16* __restrict__ in,
                                __nv_bfloat16* __restrict__ out) {
    const int h = H / 2, w = W / 2;
    const long n = long(B) * h * w * C;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int c = int(i % C);
        const long q = i / C;
        const int x = int(q % w), y = int((q / w) % h), b = int(q / (long(w) * h));
        const size_t base = ((size_t(b) * H + 2 * y) * W + 2 * x) * C + c;
        const float a = __bfloat162float(in[base]), bb = __bfloat162float(in[base + C]);
        const float cc = __bfloat162float(in[base + size_t(W) * C]), d = __bfloat162float(in[base + size_t(W) * C + C]);
        out[i] = __float2bfloat16_rn(fmaxf(fmaxf(a, bb), fmaxf(cc, d)));
    }
}

// Gradient of max pooling, added to gin: to the first of the four inputs
// equal to the max (the order torch's max_pool2d picks).
__global__ void pool_bwd_kernel(int B, int H, int W, int C, const __nv_bfloat16* __restrict__ in,
                                const __nv_bfloat16* __restrict__ out, const float* __restrict__ gout,
                                float* __restrict__ gin) {
    const int h = H / 2, w = W / 2;
    const long n = long(B) * h * w * C;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int c = int(i % C);
        const long q = i / C;
        const int x = int(q % w), y = int((q / w) % h), b = int(q / (long(w) * h));
        const size_t base = ((size_t(b) * H + 2 * y) * W + 2 * x) * C + c;
        const size_t idx[4] = {base, base + C, base + size_t(W) * C, base + size_t(W) * C + C};
        const float m = __bfloat162float(out[i]);
        bool done = false;
        for (int k = 0; k < 4; ++k) {
            const bool pick = !done && __bfloat162float(in[idx[k]]) == m;
            if (pick) gin[idx[k]] += gout[i];
            done |= pick;
        }
    }
}

// Nearest 2x upsampling into channels [offset, offset + C) of an NHWC tensor
// of `stride` channels (the first half of a concatenation).
__global__ void up_fwd_kernel(int B, int h, int w, int C, const __nv_bfloat16* __restrict__ in,
                              __nv_bfloat16* __restrict__ out, int stride, int offset) {
    const int H = 2 * h, W = 2 * w;
    const long n = long(B) * H * W * C;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int c = int(i % C);
        const long q = i / C;
        const int x = int(q % W), y = int((q / W) % H), b = int(q / (long(W) * H));
        out[q * stride + offset + c] = in[((size_t(b) * h + y / 2) * w + x / 2) * C + c];
    }
}

// Gradient of upsampling: the sum over each 2x2 block, read from channels
// [offset, offset + C) of a `stride`-channel gradient.
__global__ void up_bwd_kernel(int B, int h, int w, int C, const float* __restrict__ gout, int stride, int offset,
                              float* __restrict__ gin) {
    const int W = 2 * w;
    const long n = long(B) * h * w * C;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int c = int(i % C);
        const long q = i / C;
        const int x = int(q % w), y = int((q / w) % h), b = int(q / (long(w) * h));
        const size_t r0 = (size_t(b) * 2 * h + 2 * y) * W + 2 * x;
        gin[i] = gout[r0 * stride + offset + c] + gout[(r0 + 1) * stride + offset + c] +
                 gout[(r0 + W) * stride + offset + c] + gout[(r0 + W + 1) * stride + offset + c];
    }
}

// Copies an NHWC tensor of C channels into channels [offset, offset + C) of
// one with `stride` channels (the skip half of a concatenation), or the
// float gradient back out of it.
__global__ void copy_channels_kernel(long pixels, int C, const __nv_bfloat16* __restrict__ src,
                                     __nv_bfloat16* __restrict__ dst, int stride, int offset) {
    const long n = pixels * C;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        dst[(i / C) * stride + offset + i % C] = src[i];
}
__global__ void add_channels_kernel(long pixels, int C, const float* __restrict__ src, int stride, int offset,
                                    float* __restrict__ dst) {
    const long n = pixels * C;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        dst[i] += src[(i / C) * stride + offset + i % C];
}

// Stores the 10 guide values of a pixel, zero-padded to `stride` channels
// (a multiple of 8), as bf16 with 16-byte stores.
__device__ __forceinline__ void store_input(const float (&g)[10], __nv_bfloat16* __restrict__ d, int stride) {
    uint32_t w[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const float a = 2 * k < 10 ? g[2 * k] : 0.0f, b = 2 * k + 1 < 10 ? g[2 * k + 1] : 0.0f;
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        w[k] = *reinterpret_cast<const uint32_t*>(&h);
    }
    uint4* q = reinterpret_cast<uint4*>(d);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (8 * k < stride) q[k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
    for (int c = 32; c < stride; c += 8) q[c / 8] = make_uint4(0, 0, 0, 0);
}

// The network input from float channels (radiance 3, albedo 3, normal 3,
// depth 1 per pixel): log(1 + radiance), albedo, normal, log(1 + depth),
// zero-padded to `stride` channels, bf16.
__global__ void input_kernel(long pixels, const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, int stride) {
    for (long p = blockIdx.x * long(blockDim.x) + threadIdx.x; p < pixels; p += long(gridDim.x) * blockDim.x) {
        const float* s = src + p * 10;
        float g[10];
        for (int c = 0; c < 3; ++c) g[c] = log1pf(fmaxf(s[c], 0.0f));
        for (int c = 3; c < 9; ++c) g[c] = s[c];
        g[9] = log1pf(fmaxf(s[9], 0.0f));
        store_input(g, dst + p * stride, stride);
    }
}

// The network input for a W x H frame padded to Wp x Hp (edge pixels
// repeated): colour 3 and depth 1 from their own planes, albedo and normal
// from the renderer's 7-float guides.
__global__ void frame_input_kernel(int W, int H, int Wp, int Hp, const float* __restrict__ color,
                                   const float* __restrict__ aux7, const float* __restrict__ depth,
                                   __nv_bfloat16* __restrict__ dst, int stride) {
    const long n = long(Wp) * Hp;
    for (long p = blockIdx.x * long(blockDim.x) + threadIdx.x; p < n; p += long(gridDim.x) * blockDim.x) {
        const int x = min(int(p % Wp), W - 1), y = min(int(p / Wp), H - 1);
        const size_t q = size_t(y) * W + x;
        float g[10];
        for (int c = 0; c < 3; ++c) g[c] = log1pf(fmaxf(color[3 * q + c], 0.0f));
        for (int c = 0; c < 6; ++c) g[3 + c] = aux7[7 * q + c];
        g[9] = log1pf(fmaxf(depth[q], 0.0f));
        store_input(g, dst + p * stride, stride);
    }
}

// Radiance of the W x H frame from the network's log output over Wp x Hp.
__global__ void frame_output_kernel(int W, int H, int Wp, int stride, const float* __restrict__ pred,
                                    float* __restrict__ out) {
    const long n = long(W) * H;
    for (long p = blockIdx.x * long(blockDim.x) + threadIdx.x; p < n; p += long(gridDim.x) * blockDim.x) {
        const long q = (p / W) * Wp + p % W;
        for (int c = 0; c < 3; ++c) out[p * 3 + c] = fmaxf(expm1f(pred[q * stride + c]), 0.0f);
    }
}

// L1 loss on log radiance: pred holds log(1 + radiance) in its first 3 of
// `stride` channels. Writes d loss / d pred (into all stride channels) and
// adds the loss sum to *loss.
__global__ void l1_kernel(long pixels, int stride, const float* __restrict__ pred, const float* __restrict__ target,
                          float scale, float* __restrict__ grad, float* __restrict__ loss) {
    float local = 0;
    for (long p = blockIdx.x * long(blockDim.x) + threadIdx.x; p < pixels; p += long(gridDim.x) * blockDim.x) {
        for (int c = 0; c < stride; ++c) {
            float g = 0;
            if (c < 3) {
                const float d = pred[p * stride + c] - log1pf(fmaxf(target[p * 3 + c], 0.0f));
                local += fabsf(d);
                g = d > 0 ? scale : d < 0 ? -scale : 0.0f;
            }
            grad[p * stride + c] = g;
        }
    }
    for (int off = 16; off > 0; off >>= 1) local += __shfl_down_sync(0xffffffffu, local, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, local);
}

// Radiance from the network's log output.
__global__ void output_kernel(long pixels, int stride, const float* __restrict__ pred, float* __restrict__ out) {
    for (long p = blockIdx.x * long(blockDim.x) + threadIdx.x; p < pixels; p += long(gridDim.x) * blockDim.x)
        for (int c = 0; c < 3; ++c) out[p * 3 + c] = fmaxf(expm1f(pred[p * stride + c]), 0.0f);
}

// Adam on float master weights, refreshing their bf16 copy.
__global__ void adam_kernel(long n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, __nv_bfloat16* __restrict__ w16, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1 - b1) * gi;
        const float vi = b2 * v[i] + (1 - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (w16) w16[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void f32_to_bf16_kernel(long n, const float* __restrict__ a, __nv_bfloat16* __restrict__ b) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        b[i] = __float2bfloat16_rn(a[i]);
}

int grid1(long n) {
    const long g = (n + 255) / 256;
    return int(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

}  // namespace

namespace unet {

cudaError_t conv_fwd(const ConvShape& s, const void* in, bool in_f32, const __nv_bfloat16* w, const float* bias,
                     bool relu, void* out, bool out_f32, int out_stride, int out_offset, cudaStream_t st) {
    const long P = long(s.B) * s.H * s.W;
    const dim3 grid(unsigned((P + 127) / 128), unsigned((s.Cout + kCoTile - 1) / kCoTile));
    const size_t smem = size_t(kCoTile) * s.Cin * sizeof(float);
    if (in_f32) {
        if (out_f32)
            conv_fwd_kernel<float, float><<<grid, 128, smem, st>>>(s.B, s.H, s.W, s.Cin, s.Cout, (const float*)in, w,
                                                                   bias, relu, (float*)out, out_stride, out_offset);
        else
            conv_fwd_kernel<float, __nv_bfloat16><<<grid, 128, smem, st>>>(
                s.B, s.H, s.W, s.Cin, s.Cout, (const float*)in, w, bias, relu, (__nv_bfloat16*)out, out_stride,
                out_offset);
    } else {
        if (out_f32)
            conv_fwd_kernel<__nv_bfloat16, float><<<grid, 128, smem, st>>>(
                s.B, s.H, s.W, s.Cin, s.Cout, (const __nv_bfloat16*)in, w, bias, relu, (float*)out, out_stride,
                out_offset);
        else
            conv_fwd_kernel<__nv_bfloat16, __nv_bfloat16><<<grid, 128, smem, st>>>(
                s.B, s.H, s.W, s.Cin, s.Cout, (const __nv_bfloat16*)in, w, bias, relu, (__nv_bfloat16*)out,
                out_stride, out_offset);
    }
    return cudaGetLastError();
}

cudaError_t conv_wgrad(const ConvShape& s, const __nv_bfloat16* in, const float* dout, float* dw, float* db,
                       cudaStream_t st) {
    const long P = long(s.B) * s.H * s.W;
    const int ci_tiles = (s.Cin + 31) / 32, co_tiles = (s.Cout + kCoTile - 1) / kCoTile;
    const int base_blocks = 9 * ci_tiles * co_tiles;
    int splits = int((148 * 8 + base_blocks - 1) / base_blocks);
    const long min_px = 2048;
    if (P / splits < min_px) splits = int(P / min_px > 0 ? P / min_px : 1);
    const long per = ((P + splits - 1) / splits + 63) / 64 * 64;
    splits = int((P + per - 1) / per);
    const dim3 grid(unsigned(9 * ci_tiles), unsigned(co_tiles), unsigned(splits));
    conv_wgrad_kernel<<<grid, 256, 0, st>>>(s.B, s.H, s.W, s.Cin, s.Cout, in, dout, dw, db, per);
    return cudaGetLastError();
}

cudaError_t bias_grad(long pixels, int C, const float* g, float* db, cudaStream_t st) {
    if (C < 1 || C > 256) return cudaErrorInvalidValue;
    const long per = 4096;
    const long blocks = (pixels + per - 1) / per;
    bias_grad_kernel<<<unsigned(blocks > 0 ? blocks : 1), 256, 0, st>>>(pixels, C, g, db, per);
    return cudaGetLastError();
}

cudaError_t flip_transpose(int Cin, int Cout, const __nv_bfloat16* w, __nv_bfloat16* wt, cudaStream_t st) {
    const long n = long(Cin) * 9 * Cout;
    flip_transpose_kernel<<<grid1(n), 256, 0, st>>>(Cin, Cout, w, wt);
    return cudaGetLastError();
}

cudaError_t relu_grad(long n, const __nv_bfloat16* y, float* g, __nv_bfloat16* g16, cudaStream_t st) {
    relu_grad_kernel<<<grid1(n), 256, 0, st>>>(n, y, g, g16);
    return cudaGetLastError();
}

cudaError_t to_bf16(long n, const float* g, __nv_bfloat16* g16, cudaStream_t st) {
    to_bf16_kernel<<<grid1(n), 256, 0, st>>>(n, g, g16);
    return cudaGetLastError();
}

cudaError_t pool_fwd(int B, int H, int W, int C, const __nv_bfloat16* in, __nv_bfloat16* out, cudaStream_t st) {
    pool_fwd_kernel<<<grid1(long(B) * H * W * C / 4), 256, 0, st>>>(B, H, W, C, in, out);
    return cudaGetLastError();
}

cudaError_t pool_bwd(int B, int H, int W, int C, const __nv_bfloat16* in, const __nv_bfloat16* out,
                     const float* gout, float* gin, cudaStream_t st) {
    pool_bwd_kernel<<<grid1(long(B) * H * W * C / 4), 256, 0, st>>>(B, H, W, C, in, out, gout, gin);
    return cudaGetLastError();
}

cudaError_t up_fwd(int B, int h, int w, int C, const __nv_bfloat16* in, __nv_bfloat16* out, int stride, int offset,
                   cudaStream_t st) {
    up_fwd_kernel<<<grid1(long(B) * 4 * h * w * C), 256, 0, st>>>(B, h, w, C, in, out, stride, offset);
    return cudaGetLastError();
}

cudaError_t up_bwd(int B, int h, int w, int C, const float* gout, int stride, int offset, float* gin,
                   cudaStream_t st) {
    up_bwd_kernel<<<grid1(long(B) * h * w * C), 256, 0, st>>>(B, h, w, C, gout, stride, offset, gin);
    return cudaGetLastError();
}

cudaError_t copy_channels(long pixels, int C, const __nv_bfloat16* src, __nv_bfloat16* dst, int stride, int offset,
                          cudaStream_t st) {
    copy_channels_kernel<<<grid1(pixels * C), 256, 0, st>>>(pixels, C, src, dst, stride, offset);
    return cudaGetLastError();
}

cudaError_t add_channels(long pixels, int C, const float* src, int stride, int offset, float* dst, cudaStream_t st) {
    add_channels_kernel<<<grid1(pixels * C), 256, 0, st>>>(pixels, C, src, stride, offset, dst);
    return cudaGetLastError();
}

cudaError_t make_input(long pixels, const float* src, __nv_bfloat16* dst, int stride, cudaStream_t st) {
    input_kernel<<<grid1(pixels), 256, 0, st>>>(pixels, src, dst, stride);
    return cudaGetLastError();
}

cudaError_t frame_input(int W, int H, int Wp, int Hp, const float* color, const float* aux7, const float* depth,
                        __nv_bfloat16* dst, int stride, cudaStream_t st) {
    frame_input_kernel<<<grid1(long(Wp) * Hp), 256, 0, st>>>(W, H, Wp, Hp, color, aux7, depth, dst, stride);
    return cudaGetLastError();
}

cudaError_t frame_output(int W, int H, int Wp, int stride, const float* pred, float* out, cudaStream_t st) {
    frame_output_kernel<<<grid1(long(W) * H), 256, 0, st>>>(W, H, Wp, stride, pred, out);
    return cudaGetLastError();
}

cudaError_t l1_loss(long pixels, int stride, const float* pred, const float* target, float* grad, float* loss,
                    cudaStream_t st) {
    l1_kernel<<<grid1(pixels), 256, 0, st>>>(pixels, stride, pred, target, 1.0f / float(pixels * 3), grad, loss);
    return cudaGetLastError();
}

cudaError_t make_output(long pixels, int stride, const float* pred, float* out, cudaStream_t st) {
    output_kernel<<<grid1(pixels), 256, 0, st>>>(pixels, stride, pred, out);
    return cudaGetLastError();
}

cudaError_t adam(long n, float* w, const float* g, float* m, float* v, __nv_bfloat16* w16, float lr, int step,
                 cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, float(step)), c2 = 1.0f - powf(b2, float(step));
    adam_kernel<<<grid1(n), 256, 0, st>>>(n, w, g, m, v, w16, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

cudaError_t f32_to_bf16(long n, const float* a, __nv_bfloat16* b, cudaStream_t st) {
    f32_to_bf16_kernel<<<grid1(n), 256, 0, st>>>(n, a, b);
    return cudaGetLastError();
}

}  // namespace unet
