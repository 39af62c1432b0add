// The learned denoiser: a U-Net over 10 input channels (radiance 3, albedo 3,
// normal 3, depth 1) with four levels of 32/64/96/128 channels, two 3x3
// convolutions with ReLU per level, 2x2 max pooling down, nearest 2x
// upsampling and channel concatenation with the encoder's outputs up, and a
// final 3x3 convolution to log(1 + radiance). Activations are bfloat16 NHWC,
// accumulation and gradients float, master weights float with Adam.
//
//   level 0 (H x W)     in(32*) -> 32 -> 32 ----------------------- cat -> 32 -> 32 -> out(16*)
//   level 1 (H/2)        pool -> 64 -> 64 ---------------- cat -> 64 -> 64 -^ up
//   level 2 (H/4)          pool -> 96 -> 96 ------ cat -> 96 -> 96 -^ up
//   level 3 (H/8)            pool -> 128 -> 128 ---------^ up
//   (* padded: the 10 input channels to 32, the 3 outputs to 16)
//
// Training minimises the L1 distance of log(1 + radiance) to a high-spp
// target. The network has no counterpart in the reference, whose denoiser
// (include/denoise.hpp) is the a-trous filter; that filter is its baseline.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "../../include/photon_cuda.h"
#include "pt_host.hpp"
#include "unet.h"

namespace pt {
pt_status cuda_fail(cudaError_t e, const char* what);
}
using namespace pt;

namespace {

struct LayerDef {
    int cin, cout, level;
    bool relu;
};
// The 15 convolutions in forward order.
const LayerDef kLayers[15] = {
    {32, 32, 0, true},   {32, 32, 0, true},  {32, 64, 1, true},  {64, 64, 1, true},   {64, 96, 2, true},
    {96, 96, 2, true},   {96, 128, 3, true}, {128, 128, 3, true}, {224, 96, 2, true}, {96, 96, 2, true},
    {160, 64, 1, true},  {64, 64, 1, true},  {96, 32, 0, true},  {32, 32, 0, true},  {32, 16, 0, false}};
constexpr int kInputReal = 10, kOutStride = 16;

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t want) {
        if (want <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, want);
        if (!e) bytes = want;
        return e;
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

}  // namespace

struct pt_unet {
    int device = 0;
    size_t w_off[15], b_off[15];  // offsets of each layer's weights and bias in the parameter arrays
    size_t n_params = 0;
    DevBuf params, grads, adam_m, adam_v, params16, wt16;  // wt16: flip-transposed weights for backward
    int step = 0;
    bool use_tc = true;
    // workspace for one (B, H, W)
    int B = 0, H = 0, W = 0;
    DevBuf act[16];      // x0, a0..a13 (bf16), out (float) -- see forward()
    DevBuf pool[3];      // p0, p1, p2
    DevBuf cat[3];       // u0, u1, u2
    DevBuf gact[16];     // gradients of x0, a0..a13, out
    DevBuf g16;          // bf16 copy of the latest ReLU-masked gradient (tensor-core backward)
    DevBuf gpool[3], gcat[3];
    DevBuf loss;
    DevBuf status;
    DevBuf pad_in, pad_out;  // pt_denoise_unet's padded frames
};

namespace {

long pixels_at(const pt_unet* n, int level) { return long(n->B) * (n->H >> level) * (n->W >> level); }

// Channel count of activation i: 0 is the padded input, 1..14 the outputs of conv 0..13, 15 the output.
int act_channels(int i) { return i == 0 ? 32 : i == 15 ? kOutStride : kLayers[i - 1].cout; }
int act_level(int i) { return i == 0 ? 0 : i == 15 ? 0 : kLayers[i - 1].level; }

cudaError_t ensure_workspace(pt_unet* n, int B, int H, int W) {
    if (B == n->B && H == n->H && W == n->W) return cudaSuccess;
    n->B = B;
    n->H = H;
    n->W = W;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 16 && !e; ++i) {
        const size_t px = size_t(pixels_at(n, act_level(i))), c = size_t(act_channels(i));
        e = n->act[i].ensure(px * c * (i == 15 ? 4 : 2));
        if (!e) e = n->gact[i].ensure(px * c * 4);
    }
    size_t g16_elems = 0;
    for (int i = 1; i < 15; ++i) {
        const size_t c = size_t(pixels_at(n, act_level(i))) * act_channels(i);
        g16_elems = c > g16_elems ? c : g16_elems;
    }
    if (!e) e = n->g16.ensure(g16_elems * 2);
    const int pool_c[3] = {32, 64, 96}, cat_c[3] = {96, 160, 224};
    for (int l = 0; l < 3 && !e; ++l) {
        const size_t pp = size_t(pixels_at(n, l + 1)), pc = size_t(pixels_at(n, l));
        e = n->pool[l].ensure(pp * pool_c[l] * 2);
        if (!e) e = n->gpool[l].ensure(pp * pool_c[l] * 4);
        if (!e) e = n->cat[l].ensure(pc * cat_c[l] * 2);
        if (!e) e = n->gcat[l].ensure(pc * cat_c[l] * 4);
    }
    return e;
}

__nv_bfloat16* w16(pt_unet* n, int l) { return n->params16.as<__nv_bfloat16>() + n->w_off[l]; }
const float* bias(pt_unet* n, int l) { return n->params.as<float>() + n->b_off[l]; }

// Convolution l from `in` into `primary` (bf16 or float), with the fused
// outputs of `o` (concatenation copy or 2x upsample into out2, 2x2 max pool).
// drop_primary: the tensor-core path need not store `primary` (inference,
// where only the concatenation reads it). Without tensor cores -- or for a
// shape they do not take -- conv_fwd writes `primary` and separate kernels
// produce the fused outputs from it.
cudaError_t conv(pt_unet* n, int l, const void* in, void* primary, bool out_f32, unet::ConvOut o, bool drop_primary,
                 cudaStream_t st) {
    const LayerDef& L = kLayers[l];
    const int h = n->H >> L.level, w = n->W >> L.level;
    unet::ConvShape s{n->B, h, w, L.cin, L.cout};
    o.out = drop_primary ? nullptr : primary;
    o.stride = L.cout;
    o.offset = 0;
    if (n->use_tc) {
        const cudaError_t e = unet::conv_fwd_tc(s, static_cast<const __nv_bfloat16*>(in), w16(n, l), bias(n, l), L.relu,
                                                o, out_f32, n->status.as<unsigned int>(), st);
        if (e != cudaErrorNotSupported) return e;
    }
    cudaError_t e = unet::conv_fwd(s, in, false, w16(n, l), bias(n, l), L.relu, primary, out_f32, L.cout, 0, st);
    const __nv_bfloat16* p = static_cast<const __nv_bfloat16*>(primary);
    if (!e && o.out2)
        e = o.up2 ? unet::up_fwd(n->B, h, w, L.cout, p, o.out2, o.stride2, o.offset2, st)
                  : unet::copy_channels(long(n->B) * h * w, L.cout, p, o.out2, o.stride2, o.offset2, st);
    if (!e && o.pool) e = unet::pool_fwd(n->B, h, w, L.cout, p, o.pool, st);
    return e;
}

unet::ConvOut to_cat(pt_unet* n, int l, int up) {
    unet::ConvOut o;
    o.out2 = n->cat[l].as<__nv_bfloat16>();
    const int cat_c[3] = {96, 160, 224};
    o.stride2 = cat_c[l];
    o.offset2 = up ? 0 : cat_c[l] - kLayers[2 * l + 1].cout;  // the skip half follows the upsampled half
    o.up2 = up;
    return o;
}

// The forward pass from act[0] (the padded input) to act[15] (float, 16
// channels). The encoder's second convolution at each level also writes
// its 2x2-pooled output and its copy into the decoder's concatenation; each
// decoder level's last convolution (and the bottleneck's) writes its
// upsampled output into the next finer concatenation.
cudaError_t forward(pt_unet* n, cudaStream_t st, bool training) {
    cudaError_t e;
    auto A = [&](int i) { return n->act[i].p; };
    const bool drop = !training;
#define TRY(x) \
    if ((e = (x))) return e
    TRY(conv(n, 0, A(0), A(1), false, {}, false, st));
    unet::ConvOut o = to_cat(n, 0, 0);
    o.pool = n->pool[0].as<__nv_bfloat16>();
    TRY(conv(n, 1, A(1), A(2), false, o, false, st));
    TRY(conv(n, 2, n->pool[0].p, A(3), false, {}, false, st));
    o = to_cat(n, 1, 0);
    o.pool = n->pool[1].as<__nv_bfloat16>();
    TRY(conv(n, 3, A(3), A(4), false, o, false, st));
    TRY(conv(n, 4, n->pool[1].p, A(5), false, {}, false, st));
    o = to_cat(n, 2, 0);
    o.pool = n->pool[2].as<__nv_bfloat16>();
    TRY(conv(n, 5, A(5), A(6), false, o, false, st));
    TRY(conv(n, 6, n->pool[2].p, A(7), false, {}, false, st));
    TRY(conv(n, 7, A(7), A(8), false, to_cat(n, 2, 1), drop, st));  // level 2: [up(a7) 128 | a5 96]
    TRY(conv(n, 8, n->cat[2].p, A(9), false, {}, false, st));
    TRY(conv(n, 9, A(9), A(10), false, to_cat(n, 1, 1), drop, st));  // level 1: [up(a9) 96 | a3 64]
    TRY(conv(n, 10, n->cat[1].p, A(11), false, {}, false, st));
    TRY(conv(n, 11, A(11), A(12), false, to_cat(n, 0, 1), drop, st));  // level 0: [up(a11) 64 | a1 32]
    TRY(conv(n, 12, n->cat[0].p, A(13), false, {}, false, st));
    TRY(conv(n, 13, A(13), A(14), false, {}, false, st));
    TRY(conv(n, 14, A(14), A(15), true, {}, false, st));
    return cudaSuccess;
}

// Backward from gact[15] (d loss / d output): weight gradients into grads,
// and d loss / d input into gact[0].
cudaError_t backward(pt_unet* n, cudaStream_t st) {
    cudaError_t e;
    const int B = n->B, H = n->H, W = n->W;
    float* G = n->grads.as<float>();
    // flip-transposed bf16 weights of every layer
    for (int l = 0; l < 15; ++l)
        TRY(unet::flip_transpose(kLayers[l].cin, kLayers[l].cout, w16(n, l), n->wt16.as<__nv_bfloat16>() + n->w_off[l],
                                 st));
    for (int i = 0; i < 15; ++i) TRY(cudaMemsetAsync(n->gact[i].p, 0, n->gact[i].bytes, st));
    auto bf = [&](int i) { return n->act[i].as<__nv_bfloat16>(); };
    auto g = [&](int i) { return n->gact[i].as<float>(); };
    // One convolution's backward: weight gradients from its input and output
    // gradient, and the input gradient through the flip-transposed weights.
    // With tensor cores on, a layer's output gradient is also rounded to bf16
    // (the copy relu_back, or to_bf16 for the last layer, leaves in g16): its
    // weight gradient is a tcgen05 GEMM over pixels of that copy and the
    // layer input, and its input gradient the tcgen05 convolution of that
    // copy with the flip-transposed weights. Tensor cores off: the float
    // gradient on CUDA cores.
    __nv_bfloat16* g16 = n->use_tc ? n->g16.as<__nv_bfloat16>() : nullptr;
    auto conv_back = [&](int l, const __nv_bfloat16* in, const float* gout, bool gout16, float* gin) -> cudaError_t {
        const LayerDef& L = kLayers[l];
        const unet::ConvShape s{B, H >> L.level, W >> L.level, L.cin, L.cout};
        cudaError_t r = cudaErrorNotSupported;
        if (gout16 && g16) {
            r = unet::conv_wgrad_tc(s, in, g16, G + n->w_off[l], n->status.as<unsigned int>(), st);
            if (!r) r = unet::bias_grad(pixels_at(n, L.level), L.cout, gout, G + n->b_off[l], st);
        }
        if (r == cudaErrorNotSupported) r = unet::conv_wgrad(s, in, gout, G + n->w_off[l], G + n->b_off[l], st);
        if (r || !gin) return r;
        const unet::ConvShape t{B, H >> L.level, W >> L.level, L.cout, L.cin};
        const __nv_bfloat16* wt = n->wt16.as<__nv_bfloat16>() + n->w_off[l];
        if (gout16 && g16) {
            unet::ConvOut o;
            o.out = gin;
            o.stride = L.cin;
            r = unet::conv_fwd_tc(t, g16, wt, nullptr, false, o, true, n->status.as<unsigned int>(), st);
            if (r != cudaErrorNotSupported) return r;
        }
        return unet::conv_fwd(t, gout, true, wt, nullptr, false, gin, true, L.cin, 0, st);
    };
    auto relu_back = [&](int i) {
        return unet::relu_grad(pixels_at(n, act_level(i)) * act_channels(i), bf(i), g(i), g16, st);
    };
    if (g16) TRY(unet::to_bf16(pixels_at(n, 0) * kOutStride, g(15), g16, st));
    TRY(conv_back(14, bf(14), g(15), true, g(14)));
    TRY(relu_back(14));
    TRY(conv_back(13, bf(13), g(14), true, g(13)));
    TRY(relu_back(13));
    TRY(conv_back(12, n->cat[0].as<__nv_bfloat16>(), g(13), true, n->gcat[0].as<float>()));
    TRY(unet::up_bwd(B, H / 2, W / 2, 64, n->gcat[0].as<float>(), 96, 0, g(12), st));
    TRY(unet::add_channels(pixels_at(n, 0), 32, n->gcat[0].as<float>(), 96, 64, g(2), st));
    TRY(relu_back(12));
    TRY(conv_back(11, bf(11), g(12), true, g(11)));
    TRY(relu_back(11));
    TRY(conv_back(10, n->cat[1].as<__nv_bfloat16>(), g(11), true, n->gcat[1].as<float>()));
    TRY(unet::up_bwd(B, H / 4, W / 4, 96, n->gcat[1].as<float>(), 160, 0, g(10), st));
    TRY(unet::add_channels(pixels_at(n, 1), 64, n->gcat[1].as<float>(), 160, 96, g(4), st));
    TRY(relu_back(10));
    TRY(conv_back(9, bf(9), g(10), true, g(9)));
    TRY(relu_back(9));
    TRY(conv_back(8, n->cat[2].as<__nv_bfloat16>(), g(9), true, n->gcat[2].as<float>()));
    TRY(unet::up_bwd(B, H / 8, W / 8, 128, n->gcat[2].as<float>(), 224, 0, g(8), st));
    TRY(unet::add_channels(pixels_at(n, 2), 96, n->gcat[2].as<float>(), 224, 128, g(6), st));
    TRY(relu_back(8));
    TRY(conv_back(7, bf(7), g(8), true, g(7)));
    TRY(relu_back(7));
    TRY(conv_back(6, n->pool[2].as<__nv_bfloat16>(), g(7), true, n->gpool[2].as<float>()));
    TRY(unet::pool_bwd(B, H / 4, W / 4, 96, bf(6), n->pool[2].as<__nv_bfloat16>(), n->gpool[2].as<float>(), g(6), st));
    TRY(relu_back(6));
    TRY(conv_back(5, bf(5), g(6), true, g(5)));
    TRY(relu_back(5));
    TRY(conv_back(4, n->pool[1].as<__nv_bfloat16>(), g(5), true, n->gpool[1].as<float>()));
    TRY(unet::pool_bwd(B, H / 2, W / 2, 64, bf(4), n->pool[1].as<__nv_bfloat16>(), n->gpool[1].as<float>(), g(4), st));
    TRY(relu_back(4));
    TRY(conv_back(3, bf(3), g(4), true, g(3)));
    TRY(relu_back(3));
    TRY(conv_back(2, n->pool[0].as<__nv_bfloat16>(), g(3), true, n->gpool[0].as<float>()));
    TRY(unet::pool_bwd(B, H, W, 32, bf(2), n->pool[0].as<__nv_bfloat16>(), n->gpool[0].as<float>(), g(2), st));
    TRY(relu_back(2));
    TRY(conv_back(1, bf(1), g(2), true, g(1)));
    TRY(relu_back(1));
    TRY(conv_back(0, bf(0), g(1), true, g(0)));
#undef TRY
    return cudaSuccess;
}

// A tensor-core convolution gave up waiting (bit 0 of the status word):
// reported once, then cleared.
pt_status status_fail(pt_unet* n, cudaStream_t st) {
    cudaMemsetAsync(n->status.p, 0, 4, st);
    cudaStreamSynchronize(st);
    return fail(PT_ERR_TIMEOUT, "pt_unet: a tensor-core convolution timed out waiting for its operands");
}

pt_status check_size(int B, int H, int W, const char* what) {
    if (B < 1 || H < 8 || W < 8 || H % 8 || W % 8)
        return fail(PT_ERR_INVALID_ARG, std::string(what) + ": batch >= 1 and height, width multiples of 8 are required");
    if (long(B) * H * W > (1L << 28)) return fail(PT_ERR_INVALID_ARG, std::string(what) + ": too many pixels");
    return PT_OK;
}

}  // namespace

extern "C" {

pt_status pt_unet_create(uint64_t seed, pt_unet** out) {
    clear_error();
    if (!out) return fail(PT_ERR_INVALID_ARG, "pt_unet_create: null pointer");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PT_ERR_NO_DEVICE, "no CUDA device");
    pt_unet* n = new (std::nothrow) pt_unet();
    if (!n) return fail(PT_ERR_OUT_OF_MEMORY, "pt_unet_create: out of host memory");
    cudaGetDevice(&n->device);
    size_t off = 0;
    for (int l = 0; l < 15; ++l) {
        n->w_off[l] = off;
        off += size_t(kLayers[l].cout) * 9 * kLayers[l].cin;
        n->b_off[l] = off;
        off += size_t(kLayers[l].cout);
    }
    n->n_params = off;
    // He-normal weights (fan-in of the real input channels), zero biases.
    std::vector<float> host(off, 0.0f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> normal(0.0f, 1.0f);
    for (int l = 0; l < 15; ++l) {
        const int fan_in = 9 * (l == 0 ? kInputReal : kLayers[l].cin);
        const float sd = std::sqrt(2.0f / float(fan_in)) * (l == 14 ? 0.5f : 1.0f);
        for (size_t i = 0; i < size_t(kLayers[l].cout) * 9 * kLayers[l].cin; ++i) host[n->w_off[l] + i] = sd * normal(rng);
    }
    cudaError_t e = n->params.ensure(off * 4);
    if (!e) e = n->grads.ensure(off * 4);
    if (!e) e = n->adam_m.ensure(off * 4);
    if (!e) e = n->adam_v.ensure(off * 4);
    if (!e) e = n->params16.ensure(off * 2);
    if (!e) e = n->wt16.ensure(off * 2);
    if (!e) e = n->loss.ensure(256);
    if (!e) e = n->status.ensure(256);
    if (!e) e = cudaMemset(n->status.p, 0, 256);
    if (!e) e = cudaMemcpy(n->params.p, host.data(), off * 4, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemset(n->adam_m.p, 0, off * 4);
    if (!e) e = cudaMemset(n->adam_v.p, 0, off * 4);
    if (!e) e = unet::f32_to_bf16(long(off), n->params.as<float>(), n->params16.as<__nv_bfloat16>(), nullptr);
    if (!e) e = cudaDeviceSynchronize();
    if (e) {
        delete n;
        return cuda_fail(e, "pt_unet_create");
    }
    *out = n;
    return PT_OK;
}

pt_status pt_unet_destroy(pt_unet* n) {
    if (n) {
        cudaSetDevice(n->device);
        delete n;
    }
    return PT_OK;
}

size_t pt_unet_num_params(const pt_unet* n) { return n ? n->n_params : 0; }

pt_status pt_unet_get_params(const pt_unet* n, float* host) {
    clear_error();
    if (!n || !host) return fail(PT_ERR_INVALID_ARG, "pt_unet_get_params: null pointer");
    // a training step may still be running on a non-blocking stream, which
    // the copy below would not wait for
    cudaError_t e = cudaDeviceSynchronize();
    if (!e) e = cudaMemcpy(host, n->params.p, n->n_params * 4, cudaMemcpyDeviceToHost);
    return e ? cuda_fail(e, "pt_unet_get_params") : PT_OK;
}

pt_status pt_unet_set_params(pt_unet* n, const float* host) {
    clear_error();
    if (!n || !host) return fail(PT_ERR_INVALID_ARG, "pt_unet_set_params: null pointer");
    cudaError_t e = cudaDeviceSynchronize();  // as in pt_unet_get_params
    if (!e) e = cudaMemcpy(n->params.p, host, n->n_params * 4, cudaMemcpyHostToDevice);
    if (!e) e = unet::f32_to_bf16(long(n->n_params), n->params.as<float>(), n->params16.as<__nv_bfloat16>(), nullptr);
    if (!e) e = cudaDeviceSynchronize();
    return e ? cuda_fail(e, "pt_unet_set_params") : PT_OK;
}

pt_status pt_unet_sync(pt_unet* n, void* stream) {
    clear_error();
    if (!n) return fail(PT_ERR_INVALID_ARG, "pt_unet_sync: null pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned int status = 0;
    cudaError_t e = cudaMemcpyAsync(&status, n->status.p, 4, cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (e) return cuda_fail(e, "pt_unet_sync");
    return status ? status_fail(n, st) : PT_OK;
}

pt_status pt_unet_set_tensor_cores(pt_unet* n, int enable) {
    clear_error();
    if (!n) return fail(PT_ERR_INVALID_ARG, "pt_unet_set_tensor_cores: null pointer");
    n->use_tc = enable != 0;
    return PT_OK;
}

pt_status pt_unet_forward(pt_unet* n, int B, int H, int W, const float* d_input, float* d_output, void* stream) {
    clear_error();
    if (!n || !d_input || !d_output) return fail(PT_ERR_INVALID_ARG, "pt_unet_forward: null pointer");
    if (pt_status s = check_size(B, H, W, "pt_unet_forward")) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = ensure_workspace(n, B, H, W);
    const long px = long(B) * H * W;
    if (!e) e = unet::make_input(px, d_input, n->act[0].as<__nv_bfloat16>(), 32, st);
    if (!e) e = forward(n, st, false);
    if (!e) e = unet::make_output(px, kOutStride, n->act[15].as<float>(), d_output, st);
    return e ? cuda_fail(e, "pt_unet_forward") : PT_OK;
}

// Forward, L1 loss on log radiance and backward; the gradients stay in the
// network (pt_unet_get_grads), input gradients in d_input_grad if given.
static pt_status loss_and_grads(pt_unet* n, int B, int H, int W, const float* d_input, const float* d_target,
                                float* loss_out, cudaStream_t st) {
    cudaError_t e = ensure_workspace(n, B, H, W);
    const long px = long(B) * H * W;
    if (!e) e = unet::make_input(px, d_input, n->act[0].as<__nv_bfloat16>(), 32, st);
    if (!e) e = forward(n, st, true);
    if (!e) e = cudaMemsetAsync(n->loss.p, 0, 4, st);
    if (!e) e = unet::l1_loss(px, kOutStride, n->act[15].as<float>(), d_target, n->gact[15].as<float>(),
                              n->loss.as<float>(), st);
    if (!e) e = cudaMemsetAsync(n->grads.p, 0, n->n_params * 4, st);
    if (!e) e = backward(n, st);
    float loss = 0;
    unsigned int status = 0;
    if (!e) e = cudaMemcpyAsync(&loss, n->loss.p, 4, cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaMemcpyAsync(&status, n->status.p, 4, cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (e) return cuda_fail(e, "pt_unet: backward");
    if (status) return status_fail(n, st);
    if (loss_out) *loss_out = loss / float(px * 3);
    return PT_OK;
}

pt_status pt_unet_train_step(pt_unet* n, int B, int H, int W, const float* d_input, const float* d_target, float lr,
                             float* loss_out, void* stream) {
    clear_error();
    if (!n || !d_input || !d_target) return fail(PT_ERR_INVALID_ARG, "pt_unet_train_step: null pointer");
    if (pt_status s = check_size(B, H, W, "pt_unet_train_step")) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (pt_status s = loss_and_grads(n, B, H, W, d_input, d_target, loss_out, st)) return s;
    n->step += 1;
    cudaError_t e = unet::adam(long(n->n_params), n->params.as<float>(), n->grads.as<float>(), n->adam_m.as<float>(),
                               n->adam_v.as<float>(), n->params16.as<__nv_bfloat16>(), lr, n->step, st);
    return e ? cuda_fail(e, "pt_unet_train_step") : PT_OK;
}

pt_status pt_unet_loss_grads(pt_unet* n, int B, int H, int W, const float* d_input, const float* d_target,
                             float* loss_out, float* host_grads, float* host_input_grad) {
    clear_error();
    if (!n || !d_input || !d_target) return fail(PT_ERR_INVALID_ARG, "pt_unet_loss_grads: null pointer");
    if (pt_status s = check_size(B, H, W, "pt_unet_loss_grads")) return s;
    if (pt_status s = loss_and_grads(n, B, H, W, d_input, d_target, loss_out, nullptr)) return s;
    cudaError_t e = cudaSuccess;
    if (host_grads) e = cudaMemcpy(host_grads, n->grads.p, n->n_params * 4, cudaMemcpyDeviceToHost);
    if (!e && host_input_grad)
        e = cudaMemcpy(host_input_grad, n->gact[0].p, size_t(B) * H * W * 32 * 4, cudaMemcpyDeviceToHost);
    return e ? cuda_fail(e, "pt_unet_loss_grads") : PT_OK;
}

pt_status pt_denoise_unet(pt_unet* n, int width, int height, const float* d_color, const float* d_aux,
                          const float* d_depth, float* d_out, void* stream) {
    clear_error();
    if (!n || !d_color || !d_aux || !d_depth || !d_out) return fail(PT_ERR_INVALID_ARG, "pt_denoise_unet: null pointer");
    if (width < 1 || height < 1) return fail(PT_ERR_INVALID_ARG, "pt_denoise_unet: empty frame");
    const int Wp = (width + 7) / 8 * 8, Hp = (height + 7) / 8 * 8;
    if (pt_status s = check_size(1, Hp, Wp, "pt_denoise_unet")) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = ensure_workspace(n, 1, Hp, Wp);
    if (!e) e = unet::frame_input(width, height, Wp, Hp, d_color, d_aux, d_depth, n->act[0].as<__nv_bfloat16>(), 32, st);
    if (!e) e = forward(n, st, false);
    if (!e) e = unet::frame_output(width, height, Wp, kOutStride, n->act[15].as<float>(), d_out, st);
    return e ? cuda_fail(e, "pt_denoise_unet") : PT_OK;
}

}  // extern "C"
