"""PT_FLAG_NEE_EXTENDED on the GPU through the C ABI: renders against the
oracle's restatement of the extended light sampling, on production streams,
at the render tests' bars (|gpu - cpu| <= 1e-4 * max(1, |cpu|) on >= 97% of
pixels, image means within 1%); and the combinations it refuses."""
import numpy as np
import pytest

from test_gpu_render import assert_render_close

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pt(built):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return built


@pytest.mark.parametrize("kind,param,w,h,spp", [
    ("MESH_LIGHT", 0, 64, 36, 4), ("REF_ROOM", 0, 64, 36, 4), ("ROOM_MESH", 4, 48, 48, 4),
    ("INSTANCES", 300, 64, 36, 2), ("TEXTURED", 0, 64, 36, 3), ("REF_MATERIALS", 0, 48, 27, 4),
])
def test_extended_render_matches_oracle(pt, kind, param, w, h, spp):
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    g = pt.Generated(getattr(abi, "PT_GEN_" + kind), seed=2, param=param)
    s = pt.Scene(g)
    img, aux, rays = s.render(g.camera, w, h, spp, 10, seed=9, aux=True, mode=abi.PT_MODE_MEGAKERNEL,
                              flags=abi.PT_FLAG_NEE_EXTENDED)
    ref, raux, rrays = Oracle(g.desc).render(g.camera, w, h, spp, 10, seed=9, rng_mode=0, aux=True,
                                             flags=abi.PT_FLAG_NEE_EXTENDED)
    assert_render_close(img, ref, kind)
    assert_render_close(aux, raux, kind + " aux")
    assert abs(int(rays) - int(rrays)) <= 0.01 * int(rrays)
    # without guides the same image (the aux-free kernel form)
    img2, _, rays2 = s.render(g.camera, w, h, spp, 10, seed=9, mode=abi.PT_MODE_AUTO, flags=abi.PT_FLAG_NEE_EXTENDED)
    assert img2.tobytes() == img.tobytes() and rays2 == rays


def test_extended_flag_is_off_by_default_and_changes_the_estimate(pt):
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_MESH_LIGHT)
    s = pt.Scene(g)
    a = s.render(g.camera, 64, 36, 4, 10, seed=5)
    b = s.render(g.camera, 64, 36, 4, 10, seed=5, flags=0)
    c = s.render(g.camera, 64, 36, 4, 10, seed=5, flags=abi.PT_FLAG_NEE_EXTENDED)
    assert a[0].tobytes() == b[0].tobytes() and a[2] == b[2]
    assert a[0].tobytes() != c[0].tobytes()


def test_extended_refusals(pt):
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_MESH_LIGHT)
    s = pt.Scene(g)
    with pytest.raises(pt.PhotonError) as e:
        s.render(g.camera, 16, 16, 1, flags=abi.PT_FLAG_NEE_EXTENDED, mode=abi.PT_MODE_WAVEFRONT)
    assert e.value.status == abi.PT_ERR_UNSUPPORTED
    with pytest.raises(pt.PhotonError) as e:
        s.render(g.camera, 16, 16, 1, flags=abi.PT_FLAG_NEE_EXTENDED, rng=abi.PT_RNG_SNAPSHOT,
                 states=np.zeros((16 * 16, 4), np.uint64))
    assert e.value.status == abi.PT_ERR_UNSUPPORTED
    with pytest.raises(pt.PhotonError) as e:
        s.render(g.camera, 16, 16, 1, flags=4)
    assert e.value.status == abi.PT_ERR_INVALID_ARG
