"""Renders on the GPU through the C ABI, against the oracle and the reference.

Tolerance. The GPU computes every float in the reference's order without
contraction, but cosf/sinf (lambertian scatter, light-cone sampling) come
from CUDA's libdevice instead of glibc and may differ by an ulp or two. A
path whose direction moved by an ulp almost always hits the same surface and
its radiance moves by ~1e-6 relative; rarely it diverges (a grazing hit, a
Russian-roulette draw at the threshold). So per pixel we require
|gpu - cpu| <= 1e-4 * max(1, |cpu|) on at least 97% of pixels, and the image
means within 1e-2 relative -- both far tighter than Monte-Carlo noise.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu

RTOL = 1e-4
MIN_CLOSE = 0.97
MEAN_RTOL = 1e-2

RENDER_FIXTURES = sorted(f for f in os.listdir(GOLDEN) if f.startswith("ref_render_"))


@pytest.fixture(scope="module")
def pt(built):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return built


def close_fraction(a, b):
    return float((np.abs(a - b) <= RTOL * np.maximum(1.0, np.abs(b))).all(axis=-1).mean())


def assert_render_close(img, ref, what=""):
    frac = close_fraction(img, ref)
    m_img, m_ref = float(img.mean(dtype=np.float64)), float(ref.mean(dtype=np.float64))
    assert frac >= MIN_CLOSE, f"{what}: only {frac:.4f} of pixels within {RTOL}"
    assert abs(m_img - m_ref) <= MEAN_RTOL * max(abs(m_ref), 1e-3), f"{what}: means {m_img} vs {m_ref}"


def camera_from(arr):
    from photon_tracer_b200 import abi
    return abi.pt_camera.from_buffer_copy(np.ascontiguousarray(arr, np.float32).tobytes())


@pytest.mark.parametrize("name", RENDER_FIXTURES)
def test_snapshot_render_matches_reference(pt, name):
    """Driven by the reference's own per-row stream (states captured before
    each sample's path), the GPU render matches the reference's image."""
    from photon_tracer_b200 import abi
    f = golden(name)
    g = pt.Generated(int(f["kind"]), seed=1, param=int(f["param"]))
    s = pt.Scene(g)
    w, h, spp = int(f["width"]), int(f["height"]), int(f["spp"])
    img, aux, rays = s.render(camera_from(f["camera"]), w, h, spp, 10, seed=int(f["seed"]), rng=abi.PT_RNG_SNAPSHOT,
                              states=f["states"], aux=True, mode=abi.PT_MODE_MEGAKERNEL)
    assert_render_close(img, f["image"], name)
    assert_render_close(aux, f["aux"], name + " aux")
    assert abs(int(rays) - int(f["rays"])) <= 0.01 * int(f["rays"])


@pytest.mark.parametrize("seed", range(4))
def test_snapshot_material_renders_match_reference(pt, seed):
    """The reference's renders of random-material scenes -- metal fuzz above 1
    (clamped to 1 by its constructor), dielectric ior at and below 1, negative
    radii, emitters -- replayed on the GPU from the reference's own per-row
    stream: image, guides and ray count at the render bars."""
    from handmade import random_material_scene
    from photon_tracer_b200 import abi
    f = golden("ref_material_renders.npz")
    d, cam = random_material_scene(pt, 500 + seed)
    s = pt.Scene(d.desc_ptr)
    img, aux, rays = s.render(cam, 24, 16, 4, 10, seed=seed, rng=abi.PT_RNG_SNAPSHOT, states=f[f"s{seed}_states"],
                              aux=True, mode=abi.PT_MODE_MEGAKERNEL)
    assert_render_close(img, f[f"s{seed}_image"], f"materials {seed}")
    assert_render_close(aux, f[f"s{seed}_aux"], f"materials {seed} aux")
    assert abs(int(rays) - int(f[f"s{seed}_rays"])) <= 0.01 * int(f[f"s{seed}_rays"])
    wf = s.render(cam, 24, 16, 4, 10, seed=seed, rng=abi.PT_RNG_SNAPSHOT, states=f[f"s{seed}_states"], aux=True,
                  mode=abi.PT_MODE_WAVEFRONT)
    assert wf[0].tobytes() == img.tobytes() and wf[1].tobytes() == aux.tobytes() and wf[2] == rays


@pytest.mark.parametrize("kind,param,w,h,spp", [
    ("ROOM_MESH", 6, 64, 64, 4), ("RANDOM_SPHERES", 0, 80, 45, 4), ("INSTANCES", 0, 64, 36, 2),
    ("REF_ROOM", 0, 64, 36, 4), ("REF_MATERIALS", 0, 64, 36, 4), ("TEXTURED", 0, 64, 36, 4),
])
def test_sample_stream_render_matches_oracle(pt, kind, param, w, h, spp):
    """Production streams (one per pixel and sample): GPU vs the oracle's
    restatement of the same streams, image and aux."""
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    g = pt.Generated(getattr(abi, "PT_GEN_" + kind), seed=2, param=param)
    s = pt.Scene(g)
    img, aux, rays = s.render(g.camera, w, h, spp, 10, seed=9, aux=True, mode=abi.PT_MODE_MEGAKERNEL)
    ref, raux, rrays = Oracle(g.desc).render(g.camera, w, h, spp, 10, seed=9, rng_mode=0, aux=True)
    assert_render_close(img, ref, kind)
    assert_render_close(aux, raux, kind + " aux")
    assert abs(int(rays) - int(rrays)) <= 0.01 * int(rrays)


def test_non_finite_scenes_render_like_oracle(pt):
    """Scenes with NaN or huge triangle and sphere coordinates, flat and
    instanced (their node boxes are not all ordered, so every ray takes the
    exact SSE-emulating slab test): GPU renders against the oracle's, whose
    renders of the same scenes equal the reference's (tests/test_oracle.py)."""
    from handmade import non_finite_instances, non_finite_scene, non_finite_spheres
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    cam = pt.camera_look_at((0.0, 0.5, 6.0), (0.0, 0.0, 0.0), 50.0, 1.5)
    tris, spheres, g = non_finite_scene(pt)[0], non_finite_spheres(pt)[0], non_finite_instances(pt)[0]
    for what, scene, desc, c in (("triangles", tris.desc_ptr, tris.desc, cam),
                                 ("spheres", spheres.desc_ptr, spheres.desc, cam),
                                 ("instances", g, g.desc, g.camera)):
        s = pt.Scene(scene)
        img, aux, rays = s.render(c, 48, 32, 4, 10, seed=9, aux=True, mode=abi.PT_MODE_MEGAKERNEL)
        ref, raux, rrays = Oracle(desc).render(c, 48, 32, 4, 10, seed=9, rng_mode=0, aux=True)
        # a NaN triangle's normal is NaN in the aux guides: same pixels, then
        # the rest within the render tolerance
        assert np.array_equal(np.isnan(img), np.isnan(ref)) and np.array_equal(np.isnan(aux), np.isnan(raux))
        assert_render_close(np.nan_to_num(img), np.nan_to_num(ref), what)
        assert_render_close(np.nan_to_num(aux), np.nan_to_num(raux), what + " aux")
        assert abs(int(rays) - int(rrays)) <= 0.01 * int(rrays)


def test_render_is_deterministic_and_row_call_agrees(pt):
    """Same seed, same bytes; render_row_linear(j) equals row H-1-j of the frame."""
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_ROOM_MESH, seed=1, param=5)
    s = pt.Scene(g)
    a, ax, ra = s.render(g.camera, 96, 64, 3, 10, seed=4, aux=True)
    b, bx, rb = s.render(g.camera, 96, 64, 3, 10, seed=4, aux=True)
    assert a.tobytes() == b.tobytes() and ax.tobytes() == bx.tobytes() and ra == rb
    for j in (0, 17, 63):
        row = np.empty(3 * 96, np.float32)
        rx = np.empty(7 * 96, np.float32)
        pt.render_row_linear(s, g.camera, j, 96, 64, 3, 10, row, 4, 0, rx)
        assert row.tobytes() == a[63 - j].tobytes()
        assert rx.tobytes() == ax[63 - j].tobytes()


def test_progressive_passes_continue_the_sequence(pt):
    """first_sample continues the per-pixel sample numbering: two 4-spp passes
    average to the 8-spp frame (up to float summation order)."""
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_RANDOM_SPHERES, seed=1)
    s = pt.Scene(g)
    full, _, r8 = s.render(g.camera, 80, 45, 8, 10, seed=3)
    p0, _, r0 = s.render(g.camera, 80, 45, 4, 10, seed=3, first_sample=0)
    p1, _, r1 = s.render(g.camera, 80, 45, 4, 10, seed=3, first_sample=4)
    assert r0 + r1 == r8
    np.testing.assert_allclose((p0 + p1) / 2, full, rtol=2e-5, atol=1e-6)


def test_depth_zero_and_one(pt):
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_REF_FIELD, seed=1)
    s = pt.Scene(g)
    img, aux, rays = s.render(g.camera, 40, 23, 2, 0, seed=1, aux=True)
    assert not img.any() and not aux.any() and rays == 0
    img, aux, rays = s.render(g.camera, 40, 23, 2, 1, seed=1, aux=True)
    ref, raux, rrays = Oracle(g.desc).render(g.camera, 40, 23, 2, 1, seed=1, rng_mode=0, aux=True)
    assert_render_close(img, ref, "depth 1")
    assert rays == rrays == 40 * 23 * 2


def test_invalid_settings_are_refused(pt):
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_REF_ROOM)
    s = pt.Scene(g)
    for kw in (dict(width=1, height=10, spp=1), dict(width=10, height=10, spp=0), dict(width=10, height=10, spp=1,
                                                                                      max_bounces=-1)):
        with pytest.raises(pt.PhotonError) as e:
            s.render(g.camera, **kw)
        assert e.value.status == abi.PT_ERR_INVALID_ARG
    with pytest.raises(pt.PhotonError):
        s.render(g.camera, 10, 10, 1, rng=abi.PT_RNG_SNAPSHOT, states=None)


def block_z(image, mean, sigma, seeds, block=20, floor=2e-4):
    """tests/render_test.py:151-182 of the reference: worst |z| per block, per
    row of blocks and per image channel."""
    h, w, _ = image.shape
    bw, bh = w // block, h // block
    means = image[:bh * block, :bw * block].reshape(bh, block, bw, block, 3).mean(axis=(1, 3), dtype=np.float64)
    diffs = means.reshape(-1) - mean
    var = (np.maximum(sigma, floor) * np.sqrt(1 + 1 / seeds)) ** 2
    d3, v3 = diffs.reshape(bh, bw, 3), var.reshape(bh, bw, 3)
    return (float(np.max(np.abs(diffs) / np.sqrt(var))), float(np.max(np.abs(d3.sum(axis=1)) / np.sqrt(v3.sum(axis=1)))),
            float(np.max(np.abs(d3.sum(axis=(0, 1)) / np.sqrt(v3.sum(axis=(0, 1)))))))


@pytest.mark.parametrize("scene,gen", [("materials", "REF_MATERIALS"), ("field", "REF_FIELD"), ("room", "REF_ROOM"),
                                       ("teapot", "teapot"), ("crowd", "crowd"), ("crowd", "crowd, flattened"),
                                       ("spot_crowd", "spot_crowd")])
def test_reference_statistical_fixture(pt, scene, gen):
    """The reference's own render regression (tests/render_test.py check with
    tests/reference.json): 960x540, 200 spp, seed 1, |z| <= 10 per block,
    6 per block row, 5 per image. The OBJ scenes (the teapot; the crowd of 64
    instanced teapots; the same crowd flattened into world-space triangles,
    which must match the instanced crowd's reference -- the reference's check
    of instance transforms, normals and inverses; the textured spot crowd)
    come from fixtures of the reference's own scene descriptions."""
    from photon_tracer_b200 import abi
    from scene_fixture import FixtureScene
    f = golden("reference_blocks.npz")
    meta = json.loads(str(f["meta"]))
    if gen.startswith(("teapot", "crowd", "spot")):
        g = FixtureScene(golden(f"ref_scene_{scene}.npz"), flatten=gen.endswith("flattened"))
        s = pt.Scene(g.desc_ptr)
    else:
        g = pt.Generated(getattr(abi, "PT_GEN_" + gen))
        s = pt.Scene(g)
    w = meta["width"]
    img, _, _ = s.render(g.camera, w, int(w / (16 / 9)), meta["spp"], 10, seed=1)
    b, r, i = block_z(img, f[f"{scene}_mean"], f[f"{scene}_sigma"], meta["seeds"])
    assert b <= 10 and r <= 6 and i <= 5, (gen, b, r, i)


def test_denoise_matches_oracle(pt):
    """The GPU a-trous filter against the oracle's restatement of denoise.hpp."""
    from oracle.oracle import oracle_denoise
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_REF_ROOM)
    s = pt.Scene(g)
    img, aux, _ = s.render(g.camera, 160, 90, 4, 10, seed=2, aux=True)
    albedo, normal = aux[..., 0:3], aux[..., 3:6]
    lum = 0.2126 * img[..., 0] + 0.7152 * img[..., 1] + 0.0722 * img[..., 2]
    variance = ((aux[..., 6] - lum * lum) / 4).astype(np.float32)
    got = pt.denoise_atrous(img, albedo, normal, variance)
    want = oracle_denoise(img, albedo, normal, variance)
    np.testing.assert_allclose(got, want, rtol=1e-3, atol=1e-5)


@pytest.mark.parametrize("kind,param,w,h,spp,aux", [
    ("ROOM_MESH", 6, 96, 64, 4, True), ("RANDOM_SPHERES", 0, 80, 45, 3, False), ("INSTANCES", 0, 64, 36, 2, True),
    ("REF_MATERIALS", 0, 50, 30, 5, True), ("TEXTURED", 0, 64, 36, 3, True),
])
def test_wavefront_equals_megakernel(pt, kind, param, w, h, spp, aux):
    """The wavefront stages run the same per-slot arithmetic in the same order
    as the megakernel lanes: identical bytes, identical ray count."""
    from photon_tracer_b200 import abi
    g = pt.Generated(getattr(abi, "PT_GEN_" + kind), seed=3, param=param)
    s = pt.Scene(g)
    a, ax, ra = s.render(g.camera, w, h, spp, 10, seed=5, aux=aux, mode=abi.PT_MODE_MEGAKERNEL)
    b, bx, rb = s.render(g.camera, w, h, spp, 10, seed=5, aux=aux, mode=abi.PT_MODE_WAVEFRONT)
    assert a.tobytes() == b.tobytes() and ra == rb
    if aux:
        assert ax.tobytes() == bx.tobytes()


def test_wavefront_snapshot_and_depth_zero(pt):
    from photon_tracer_b200 import abi
    f = golden("ref_render_room_mesh.npz")
    g = pt.Generated(int(f["kind"]), seed=1, param=int(f["param"]))
    s = pt.Scene(g)
    w, h, spp = int(f["width"]), int(f["height"]), int(f["spp"])
    kw = dict(seed=int(f["seed"]), rng=abi.PT_RNG_SNAPSHOT, states=f["states"], aux=True)
    a = s.render(camera_from(f["camera"]), w, h, spp, 10, mode=abi.PT_MODE_MEGAKERNEL, **kw)
    b = s.render(camera_from(f["camera"]), w, h, spp, 10, mode=abi.PT_MODE_WAVEFRONT, **kw)
    assert a[0].tobytes() == b[0].tobytes() and a[1].tobytes() == b[1].tobytes() and a[2] == b[2]
    img, ax, rays = s.render(g.camera, 40, 30, 2, 0, seed=1, aux=True, mode=abi.PT_MODE_WAVEFRONT)
    assert not img.any() and not ax.any() and rays == 0
