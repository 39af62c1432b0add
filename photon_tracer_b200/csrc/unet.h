// Internal interface of the U-Net denoiser's kernels (unet_kernels.cu,
// unet_tc.cu) for the network code (unet.cpp).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace unet {

struct ConvShape {
    int B, H, W, Cin, Cout;
};

// out[.., out_offset + co] (row stride out_stride) = act(bias + conv3x3(in, w)), padding 1.
cudaError_t conv_fwd(const ConvShape& s, const void* in, bool in_f32, const __nv_bfloat16* w, const float* bias,
                     bool relu, void* out, bool out_f32, int out_stride, int out_offset, cudaStream_t st);
// dw += d loss / d w, db += d loss / d bias, from the layer input and the gradient of its output.
cudaError_t conv_wgrad(const ConvShape& s, const __nv_bfloat16* in, const float* dout, float* dw, float* db,
                       cudaStream_t st);
// db[c] += sum over pixels of g[p][c], g NHWC float with C <= 256 channels.
cudaError_t bias_grad(long pixels, int C, const float* g, float* db, cudaStream_t st);
cudaError_t flip_transpose(int Cin, int Cout, const __nv_bfloat16* w, __nv_bfloat16* wt, cudaStream_t st);
cudaError_t relu_grad(long n, const __nv_bfloat16* y, float* g, __nv_bfloat16* g16, cudaStream_t st);
cudaError_t to_bf16(long n, const float* g, __nv_bfloat16* g16, cudaStream_t st);
cudaError_t pool_fwd(int B, int H, int W, int C, const __nv_bfloat16* in, __nv_bfloat16* out, cudaStream_t st);
cudaError_t pool_bwd(int B, int H, int W, int C, const __nv_bfloat16* in, const __nv_bfloat16* out,
                     const float* gout, float* gin, cudaStream_t st);
cudaError_t up_fwd(int B, int h, int w, int C, const __nv_bfloat16* in, __nv_bfloat16* out, int stride, int offset,
                   cudaStream_t st);
cudaError_t up_bwd(int B, int h, int w, int C, const float* gout, int stride, int offset, float* gin,
                   cudaStream_t st);
cudaError_t copy_channels(long pixels, int C, const __nv_bfloat16* src, __nv_bfloat16* dst, int stride, int offset,
                          cudaStream_t st);
cudaError_t add_channels(long pixels, int C, const float* src, int stride, int offset, float* dst, cudaStream_t st);
cudaError_t make_input(long pixels, const float* src, __nv_bfloat16* dst, int stride, cudaStream_t st);
cudaError_t frame_input(int W, int H, int Wp, int Hp, const float* color, const float* aux7, const float* depth,
                        __nv_bfloat16* dst, int stride, cudaStream_t st);
cudaError_t frame_output(int W, int H, int Wp, int stride, const float* pred, float* out, cudaStream_t st);
cudaError_t l1_loss(long pixels, int stride, const float* pred, const float* target, float* grad, float* loss,
                    cudaStream_t st);
cudaError_t make_output(long pixels, int stride, const float* pred, float* out, cudaStream_t st);
cudaError_t adam(long n, float* w, const float* g, float* m, float* v, __nv_bfloat16* w16, float lr, int step,
                 cudaStream_t st);
cudaError_t f32_to_bf16(long n, const float* a, __nv_bfloat16* b, cudaStream_t st);

// Where the tensor-core convolution writes its result (any pointer may be
// null): out[p * stride + offset + co] (bf16, or float for out_f32); a bf16
// copy into out2 at the same pixel, or (up2) at the four pixels of the 2x
// finer level it covers -- the halves of a decoder's concatenation; and the
// 2x2 max pool of the result into pool ([pixel][Cout], bf16).
struct ConvOut {
    void* out = nullptr;
    int stride = 0, offset = 0;
    __nv_bfloat16* out2 = nullptr;
    int stride2 = 0, offset2 = 0, up2 = 0;
    __nv_bfloat16* pool = nullptr;
};

// Tensor-core forward convolution (tcgen05, accumulators in TMEM). Returns
// cudaErrorNotSupported for shapes it does not take (Cin % 32, Cout % 16 or
// Cout > 256; odd sizes with pool), which then run on conv_fwd.
cudaError_t conv_fwd_tc(const ConvShape& s, const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias,
                        bool relu, const ConvOut& o, bool out_f32, unsigned int* status, cudaStream_t st);

// Tensor-core weight gradient (tcgen05, MN-major operands): dw += d loss /
// d w from the layer input and the bf16 gradient of its output (Cout <= 128,
// Cin <= 256, both multiples of 8), float atomics. cudaErrorNotSupported for
// other shapes, which then run on conv_wgrad.
cudaError_t conv_wgrad_tc(const ConvShape& s, const __nv_bfloat16* in, const __nv_bfloat16* dout, float* dw,
                          unsigned int* status, cudaStream_t st);

}  // namespace unet
