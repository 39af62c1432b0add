"""Progressive rendering (pt_render_progressive): batches of growing spp
that continue the per-pixel sample numbering, summed in FP64. The samples
are the ones a single render of the full spp draws, so the image equals that
render up to the rounding of the per-batch averages."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pt(built):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return built


def test_progressive_equals_single_render(pt):
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_ROOM_MESH, seed=2, param=4)
    s = pt.Scene(g)
    st = pt.Scene.settings(160, 120, 200, 10, 5, 0, abi.PT_MODE_MEGAKERNEL, abi.PT_RNG_SAMPLE)
    calls = []
    img, done, rays = s.render_progressive(g.camera, st, lambda d, t: calls.append((d, t)) and False)
    ref, _, ref_rays = s.render(g.camera, 160, 120, 200, 10, seed=5, mode=abi.PT_MODE_MEGAKERNEL)
    assert done == 200 and rays == ref_rays
    assert calls and all(t == 200 for _, t in calls) and [d for d, _ in calls] == sorted(d for d, _ in calls)
    assert calls[0][0] == 1  # the first batch is one sample
    np.testing.assert_allclose(img, ref, rtol=2e-5, atol=1e-6)


def test_progressive_stops_when_asked(pt):
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_RANDOM_SPHERES, seed=1)
    s = pt.Scene(g)
    st = pt.Scene.settings(200, 112, 64, 10, 3, 0, abi.PT_MODE_MEGAKERNEL, abi.PT_RNG_SAMPLE)
    img, done, _ = s.render_progressive(g.camera, st, lambda d, t: True)
    one, _, _ = s.render(g.camera, 200, 112, 1, 10, seed=3, mode=abi.PT_MODE_MEGAKERNEL)
    assert done == 1
    np.testing.assert_array_equal(img, one)
