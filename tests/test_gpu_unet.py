"""The learned denoiser on the GPU, against a plain PyTorch fp32 restatement
(tests/unet_torch_ref.py) with the same weights, and the depth guide against
the library's closest-hit query.

Tolerance. Both sides round the input, the weights and every activation but
the last to bfloat16 and accumulate in fp32, but in different orders; a sum
that lands within an fp32 ulp of a bfloat16 rounding boundary rounds the
other way (a 2^-8 relative step) and the difference propagates through up
to 14 layers. So outputs and gradients are compared as whole tensors:
relative L2 error <= 3e-2 and cosine similarity >= 0.999 per layer, loss
within 1e-3 relative. (Measured on B200: 0.6% between the tensor-core and
CUDA-core forwards, up to 2.1% on the input gradient; a layout or padding
fault in a convolution gives errors of order 1.)
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_L2 = 3e-2
MIN_COS = 0.999


@pytest.fixture(scope="module")
def pt(built):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return built


def guides(rng, B, H, W):
    rad = rng.exponential(0.5, (B, H, W, 3)) * (rng.random((B, H, W, 1)) < 0.9)
    albedo = rng.random((B, H, W, 3))
    n = rng.normal(size=(B, H, W, 3))
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    depth = rng.random((B, H, W, 1)) * 8
    return np.concatenate([rad, albedo, n, depth], -1).astype(np.float32)


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def cosine(a, b):
    a, b = a.ravel().astype(np.float64), b.ravel().astype(np.float64)
    return float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-300))


def perturbed(net, rng):
    """The network's initial weights with random biases (so every term is exercised)."""
    from photon_tracer_b200.unet import param_layout
    p = net.params()
    for _, _, b_off, co in param_layout()[0]:
        p[b_off:b_off + co] = rng.normal(0, 0.05, co)
    net.set_params(p)
    return p


@pytest.mark.parametrize("tc", [False, True])
def test_unet_loss_and_gradients_match_torch(pt, tc):
    import torch
    import unet_torch_ref as ref
    from photon_tracer_b200.unet import UNet, param_layout
    rng = np.random.default_rng(3)
    B, H, W = 2, 32, 24
    # A target far above every prediction fixes the sign of each L1 term, so
    # the gradients do not hinge on predictions that sit within rounding of
    # the target (a sign flip there is a 2/(3N) jump, not a numerical error).
    x, target = guides(rng, B, H, W), np.full((B, H, W, 3), 1e4, np.float32)
    net = UNet(seed=5)
    net.tensor_cores(tc)
    p = perturbed(net, rng)
    loss, g, gi = net.loss_grads(torch.tensor(x, device="cuda"), torch.tensor(target, device="cuda"))
    r_loss, r_g, r_gi, _ = ref.loss_and_grads(p, x, target)
    assert abs(loss - r_loss) <= 1e-3 * r_loss, (loss, r_loss)
    for i, (w_off, shape, b_off, co) in enumerate(param_layout()[0]):
        n = int(np.prod(shape))
        gw, rw = g[w_off:w_off + n], r_g[w_off:w_off + n]
        if i == 14:  # only the 3 real outputs of the last layer get gradients
            gw = gw.reshape(shape)[:3]
            rw = rw.reshape(shape)[:3]
            assert not g[w_off:w_off + n].reshape(shape)[3:].any()
        assert rel_l2(gw, rw) <= REL_L2 and cosine(gw, rw) >= MIN_COS, f"layer {i} weights"
        gb, rb = g[b_off:b_off + co][:3 if i == 14 else co], r_g[b_off:b_off + co][:3 if i == 14 else co]
        assert rel_l2(gb, rb) <= REL_L2 and cosine(gb, rb) >= MIN_COS, f"layer {i} bias"
    assert rel_l2(gi, r_gi) <= REL_L2 and cosine(gi, r_gi) >= MIN_COS


@pytest.mark.parametrize("tc", [False, True])
def test_unet_forward_matches_torch(pt, tc):
    import torch
    import unet_torch_ref as ref
    from photon_tracer_b200.unet import UNet
    rng = np.random.default_rng(4)
    B, H, W = 3, 40, 32
    x = guides(rng, B, H, W)
    net = UNet(seed=6)
    net.tensor_cores(tc)
    p = perturbed(net, rng)
    out = net.forward(torch.tensor(x, device="cuda")).cpu().numpy()
    _, _, _, r_out = ref.loss_and_grads(p, x, np.zeros((B, H, W, 3), np.float32))
    assert rel_l2(out, r_out) <= REL_L2 and cosine(out, r_out) >= MIN_COS


def test_tensor_core_forward_matches_cuda_cores(pt):
    """The tcgen05 convolutions against the CUDA-core ones on the same bf16
    inputs: only the summation order differs."""
    import torch
    from photon_tracer_b200.unet import UNet
    rng = np.random.default_rng(8)
    B, H, W = 2, 64, 48
    x = torch.tensor(guides(rng, B, H, W), device="cuda")
    net = UNet(seed=9)
    perturbed(net, rng)
    net.tensor_cores(False)
    a = net.forward(x).cpu().numpy()
    net.tensor_cores(True)
    b = net.forward(x).cpu().numpy()
    assert rel_l2(b, a) <= 1.5e-2 and cosine(b, a) >= 0.9999


def test_unet_training_reduces_loss(pt):
    import torch
    from photon_tracer_b200.unet import UNet
    rng = np.random.default_rng(5)
    B, H, W = 4, 32, 32
    x = guides(rng, B, H, W)
    target = (x[..., 0:3] * 0.5 + 0.1 * x[..., 3:6]).astype(np.float32)  # learnable from the guides
    xd, td = torch.tensor(x, device="cuda"), torch.tensor(target, device="cuda")
    net = UNet(seed=1)
    losses = [net.train_step(xd, td, 1e-3) for _ in range(60)]
    assert np.isfinite(losses).all()
    assert np.mean(losses[-5:]) < 0.5 * np.mean(losses[:5]), losses


def test_denoise_frame_pads_and_crops(pt):
    """pt_denoise_unet on a frame that is not a multiple of 8 equals the
    batched forward on the edge-repeated padded frame, cropped."""
    import torch
    from photon_tracer_b200.unet import UNet
    rng = np.random.default_rng(6)
    H, W = 29, 37
    g = guides(rng, 1, H, W)[0]
    color = torch.tensor(g[..., 0:3], device="cuda").contiguous()
    aux = torch.tensor(np.concatenate([g[..., 3:9], rng.random((H, W, 1))], -1).astype(np.float32), device="cuda")
    depth = torch.tensor(g[..., 9], device="cuda").contiguous()
    net = UNet(seed=2)
    out = net.denoise(color, aux, depth).cpu().numpy()
    padded = np.pad(g, ((0, 32 - H), (0, 40 - W), (0, 0)), mode="edge")[None]
    full = net.forward(torch.tensor(np.ascontiguousarray(padded), device="cuda")).cpu().numpy()[0]
    np.testing.assert_array_equal(out, full[:H, :W])


def test_primary_depth_matches_closest_hit(pt):
    """The depth guide is t * |d| of the closest hit along each pixel's centre
    ray; the same rays through pt_trace_closest give bit-identical values."""
    from photon_tracer_b200 import abi
    from photon_tracer_b200.unet import primary_depth
    g = pt.Generated(abi.PT_GEN_REF_ROOM)
    s = pt.Scene(g)
    W, H = 64, 48
    cam = g.camera
    depth = primary_depth(s, cam, W, H).cpu().numpy()
    f32 = np.float32
    org, llc = np.array(cam.origin, f32), np.array(cam.lower_left, f32)
    hor, ver = np.array(cam.horizontal, f32), np.array(cam.vertical, f32)
    j, i = np.mgrid[0:H, 0:W]
    u = ((i.astype(f32) + f32(0.5)) / f32(W - 1)).astype(f32)[..., None]
    v = ((j.astype(f32) + f32(0.5)) / f32(H - 1)).astype(f32)[..., None]
    d = (((llc + hor * u) + ver * v) - org).astype(f32)
    rays = np.concatenate([np.broadcast_to(org, d.shape), d], -1).reshape(-1, 6)
    hits = s.trace_closest(rays)
    dd = d.reshape(-1, 3)
    norm = np.sqrt(((dd[:, 0] * dd[:, 0] + dd[:, 1] * dd[:, 1]) + dd[:, 2] * dd[:, 2]).astype(f32))
    want = np.where(hits["kind"] == abi.PT_HIT_NONE, f32(0), (hits["t"] * norm).astype(f32)).reshape(H, W)
    assert (want > 0).mean() > 0.5
    np.testing.assert_array_equal(depth, want[::-1])
