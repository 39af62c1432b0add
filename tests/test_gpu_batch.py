"""Batched rendering (pt_batch_*): scenes of different size, resolution and
spp in one arena. Every strategy must give each scene exactly the image a
single-scene render gives (same per-pixel streams, same order of sums)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pt(built):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return built


def small_batch(pt):
    """Mixed scenes at small sizes: batch-generator scenes plus instances, the reference room and two textured rooms."""
    from photon_tracer_b200 import abi
    items = []
    for s in (3, 7, 12, 21):
        g = pt.Generated(abi.PT_GEN_BATCH_SCENE, seed=s)
        items.append((g, g.camera, 48 + 8 * s, 40 + 4 * s, 2 + s % 3, 100 + s))
    g = pt.Generated(abi.PT_GEN_INSTANCES, seed=2, param=300)
    items.append((g, g.camera, 64, 36, 2, 5))
    g = pt.Generated(abi.PT_GEN_REF_ROOM)
    items.append((g, g.camera, 50, 30, 3, 9))
    for s in (4, 5):  # textures: their numbers and texel offsets are rebased in the merged arena
        g = pt.Generated(abi.PT_GEN_TEXTURED, seed=s)
        items.append((g, g.camera, 56, 32, 2, 30 + s))
    return items


@pytest.mark.parametrize("strategy", ["ONE_LAUNCH", "PER_SCENE_MEGA", "PER_SCENE_WAVE", "AUTO"])
def test_batch_matches_single_renders(pt, strategy):
    from photon_tracer_b200 import abi
    items = small_batch(pt)
    b = pt.Batch(items, getattr(abi, "PT_BATCH_" + strategy))
    rays = b.render()
    total = 0
    for i, (g, cam, w, h, spp, seed) in enumerate(items):
        img, _, r = pt.Scene(g).render(cam, w, h, spp, 10, seed=seed, mode=abi.PT_MODE_MEGAKERNEL)
        total += r
        assert b.image(i).tobytes() == img.tobytes(), f"scene {i}"
    assert rays == total
    times = b.scene_times()
    assert np.all(times > 0) and np.all(np.isfinite(times))
    info = b.info()
    assert info.n_scenes == len(items) and info.total_pixels == sum(w * h for _, _, w, h, _, _ in items)
    if strategy == "AUTO":
        assert info.tuned == 1 and min(info.tune_ms[:7]) > 0


def test_batch_replay_is_deterministic(pt):
    from photon_tracer_b200 import abi
    b = pt.Batch(small_batch(pt), abi.PT_BATCH_ONE_LAUNCH)
    r1 = b.render()
    a = [b.image(i) for i in range(6)]
    r2 = b.render()
    assert r1 == r2 and all(b.image(i).tobytes() == a[i].tobytes() for i in range(6))


def test_batch_refuses_bad_items(pt):
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_REF_MATERIALS)  # no BVH by default: refused
    with pytest.raises(pt.PhotonError) as e:
        pt.Batch([(g, g.camera, 32, 32, 1, 1)])
    assert e.value.status == abi.PT_ERR_UNSUPPORTED


@pytest.mark.parametrize("strategy", ["ONE_LAUNCH", "PER_SCENE_MEGA"])
def test_download_waits_for_a_render_on_the_callers_stream(pt, strategy):
    """render(count_rays=False) on a caller's stream returns without waiting;
    the download that follows must still see the finished images."""
    import torch
    from photon_tracer_b200 import abi
    items = small_batch(pt)
    want = pt.Batch(items, getattr(abi, "PT_BATCH_" + strategy))
    want.render()
    ref = [want.image(i) for i in range(len(items))]
    b = pt.Batch(items, getattr(abi, "PT_BATCH_" + strategy))
    s = torch.cuda.Stream()
    b.render(stream=s.cuda_stream, count_rays=False)
    assert all(b.image(i).tobytes() == ref[i].tobytes() for i in range(len(items)))
    assert np.all(np.isfinite(b.scene_times()))
