"""pt_denoise_atrous_device_noalloc: the a-trous filter for callers that
cannot allocate device memory -- a host that owns all device memory through
its own pool, or a frame loop where cudaMalloc (which can synchronise and can
fail) is not allowed. It takes its scratch from a fixed array inside the
library instead of a caller-provided buffer.

Called through the C ABI on device buffers and checked against the
entry point that takes the caller's scratch, on two calls in a row (the
second on different data, so stale contents of the shared array would show).
This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def frame(seed):
    """A rendered frame with its guides: color, albedo, normal, variance (device tensors)."""
    import torch
    import photon_tracer_b200 as pt
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_REF_ROOM)
    s = pt.Scene(g)
    w, h, spp = 320, 180, 4
    img, aux, _ = s.render(g.camera, w, h, spp, 10, seed=seed, aux=True)
    lum = 0.2126 * img[..., 0] + 0.7152 * img[..., 1] + 0.0722 * img[..., 2]
    var = ((aux[..., 6] - lum * lum) / spp).astype(np.float32)
    arrays = [img, aux[..., 0:3], aux[..., 3:6], var]
    return w, h, [torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda() for a in arrays]


def test_noalloc_matches_scratch_entry_point(built):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    lib = built.load()
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (11, 12):
        w, h, (color, albedo, normal, variance) = frame(seed)
        ptrs = [C.c_void_p(t.data_ptr()) for t in (color, albedo, normal, variance)]
        scratch = torch.empty(lib.pt_denoise_atrous_scratch_floats(w, h), dtype=torch.float32, device="cuda")
        want = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
        got = torch.full((h, w, 3), float("nan"), dtype=torch.float32, device="cuda")
        st = lib.pt_denoise_atrous_device(w, h, *ptrs, C.c_void_p(want.data_ptr()), C.c_void_p(scratch.data_ptr()),
                                          C.c_void_p(stream))
        assert st == 0, lib.pt_last_error()
        st = lib.pt_denoise_atrous_device_noalloc(w, h, *ptrs, C.c_void_p(got.data_ptr()), C.c_void_p(stream))
        assert st == 0, lib.pt_last_error()
        torch.cuda.synchronize()
        g, wnt = got.cpu().numpy(), want.cpu().numpy()
        assert np.isfinite(g).all()
        # same kernels on the same inputs: the tolerance of the denoiser tests
        np.testing.assert_allclose(g, wnt, rtol=1e-3, atol=1e-5)


@pytest.mark.parametrize("w,h", [(512, 512), (1024, 256)])
def test_noalloc_at_its_pixel_limit(built, w, h):
    """Frames of exactly PT_ATROUS_NOALLOC_MAX_PIXELS pixels fill the whole
    built-in array: seeded random guides, against caller-owned scratch."""
    import torch
    from photon_tracer_b200 import abi
    assert w * h == abi.PT_ATROUS_NOALLOC_MAX_PIXELS
    lib = built.load()
    stream = torch.cuda.current_stream().cuda_stream
    gen = torch.Generator(device="cuda").manual_seed(w)
    color = torch.rand((h, w, 3), device="cuda", generator=gen) * 3
    albedo = torch.rand((h, w, 3), device="cuda", generator=gen)
    normal = torch.randn((h, w, 3), device="cuda", generator=gen)
    variance = torch.rand((h, w), device="cuda", generator=gen)
    ptrs = [C.c_void_p(t.data_ptr()) for t in (color, albedo, normal, variance)]
    scratch = torch.empty(lib.pt_denoise_atrous_scratch_floats(w, h), dtype=torch.float32, device="cuda")
    want = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
    got = torch.full((h, w, 3), float("nan"), dtype=torch.float32, device="cuda")
    assert lib.pt_denoise_atrous_device(w, h, *ptrs, C.c_void_p(want.data_ptr()), C.c_void_p(scratch.data_ptr()),
                                        C.c_void_p(stream)) == 0, lib.pt_last_error()
    assert lib.pt_denoise_atrous_device_noalloc(w, h, *ptrs, C.c_void_p(got.data_ptr()), C.c_void_p(stream)) == 0, \
        lib.pt_last_error()
    torch.cuda.synchronize()
    g, wnt = got.cpu().numpy(), want.cpu().numpy()
    assert np.isfinite(g).all()
    np.testing.assert_allclose(g, wnt, rtol=1e-3, atol=1e-5)


def test_noalloc_refuses_frames_beyond_its_scratch(built):
    import torch
    from photon_tracer_b200 import abi
    lib = built.load()
    x = torch.zeros(16, dtype=torch.float32, device="cuda")
    p = C.c_void_p(x.data_ptr())
    st = lib.pt_denoise_atrous_device_noalloc(513, 512, p, p, p, p, p, None)
    assert st == abi.PT_ERR_INVALID_ARG
    assert b"262144" in lib.pt_last_error()
