"""Pins the CPU oracle (the C restatement) before anything is checked against
it: against the reference's golden vectors committed under tests/golden/,
against the reference itself (oracle/_ref) where it was built, and against
the reference's own statistical fixture. Also checks that the scene
generators reproduce the reference's scenes and constructors. CPU only."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden

HIT_FIXTURES = sorted(f for f in os.listdir(GOLDEN) if f.startswith("ref_hits_"))
RENDER_FIXTURES = sorted(f for f in os.listdir(GOLDEN) if f.startswith("ref_render_"))


def camera_from(arr):
    from photon_tracer_b200 import abi
    return abi.pt_camera.from_buffer_copy(np.ascontiguousarray(arr, np.float32).tobytes())


@pytest.mark.parametrize("name", HIT_FIXTURES)
def test_oracle_hits_match_reference_fixture(built, name):
    from oracle.oracle import Oracle
    f = golden(name)
    g = built.Generated(int(f["kind"]), seed=1, param=int(f["param"]))
    o = Oracle(g.desc)
    hits = o.trace_closest(f["rays"])
    assert np.array_equal(hits.view(np.uint32).reshape(-1, 6), f["hits"])
    assert np.array_equal(o.trace_any(f["rays"]), f["occluded"])


@pytest.mark.parametrize("name", RENDER_FIXTURES)
def test_oracle_renders_match_reference_fixture(built, name):
    """Per-row stream and snapshot mode both reproduce the reference's floats."""
    from oracle.oracle import Oracle
    f = golden(name)
    g = built.Generated(int(f["kind"]), seed=1, param=int(f["param"]))
    o = Oracle(g.desc)
    cam = camera_from(f["camera"])
    w, h, spp, seed = int(f["width"]), int(f["height"]), int(f["spp"]), int(f["seed"])
    img, aux, rays = o.render(cam, w, h, spp, 10, seed=seed, rng_mode=2, aux=True)
    assert img.tobytes() == f["image"].tobytes()
    assert aux.tobytes() == f["aux"].tobytes()
    assert rays == int(f["rays"])
    img2, aux2, rays2 = o.render(cam, w, h, spp, 10, seed=seed, rng_mode=1, states=f["states"], aux=True)
    assert img2.tobytes() == f["image"].tobytes() and rays2 == rays


def test_oracle_matches_reference_live(built):
    from oracle.oracle import Oracle, Reference, ref_available
    if not ref_available():
        pytest.skip("reference harness absent")
    from photon_tracer_b200 import abi
    for kind, param, seed in [(abi.PT_GEN_ROOM_MESH, 3, 11), (abi.PT_GEN_REF_MATERIALS, 0, 1),
                              (abi.PT_GEN_INSTANCES, 150, 4), (abi.PT_GEN_BATCH_SCENE, 0, 23),
                              (abi.PT_GEN_TEXTURED, 0, 7)]:
        g = built.Generated(kind, seed=seed, param=param)
        o, r = Oracle(g.desc), Reference(g.desc)
        rays = built.generate_rays(seed, [-4, -1, -4], [4, 3, 4], 5000)
        ho = o.trace_closest(rays)
        hr, bad = r.trace_closest(rays)
        assert bad == 0 and ho.tobytes() == hr.tobytes()
        assert np.array_equal(o.trace_any(rays, 0.001, 3.0), r.trace_any(rays, 0.001, 3.0))
        io, ao, ro = o.render(g.camera, 24, 16, 3, 10, seed=seed, rng_mode=2, aux=True, first_sample=5)
        ir, ar, rr = r.render(g.camera, 24, 16, 3, 10, seed=seed, aux=True, first_sample=5)
        assert io.tobytes() == ir.tobytes() and ao.tobytes() == ar.tobytes() and ro == rr


def test_oracle_no_bvh_matches_reference(built):
    """The reference's plain-list mode (geometry::build(false)) is the default for materials."""
    from oracle.oracle import Oracle, Reference, ref_available
    if not ref_available():
        pytest.skip("reference harness absent")
    from photon_tracer_b200 import abi
    g = built.Generated(abi.PT_GEN_REF_FIELD, seed=1, use_bvh=0)
    o, r = Oracle(g.desc), Reference(g.desc)
    rays = built.generate_rays(3, [-3, -0.5, -3], [3, 2, 1], 4000)
    assert o.trace_closest(rays).tobytes() == r.trace_closest(rays)[0].tobytes()


def test_oracle_random_render_settings_match_reference(built):
    """Renders through the reference's per-row stream over random settings:
    frame sizes down to 1x1, depth 0 to 11, 1 to 5 spp, sample offsets, five
    scene families."""
    from oracle.oracle import Oracle, Reference, ref_available
    if not ref_available():
        pytest.skip("reference harness absent")
    from photon_tracer_b200 import abi
    rng = np.random.default_rng(11)
    scenes = [(abi.PT_GEN_ROOM_MESH, 3), (abi.PT_GEN_REF_MATERIALS, 0), (abi.PT_GEN_INSTANCES, 40),
              (abi.PT_GEN_RANDOM_SPHERES, 0), (abi.PT_GEN_TEXTURED, 0)]
    for trial in range(15):
        kind, param = scenes[trial % len(scenes)]
        g = built.Generated(kind, seed=int(rng.integers(1, 50)), param=param)
        w, h = int(rng.integers(1, 20)), int(rng.integers(1, 14))
        spp, depth = int(rng.integers(1, 6)), int(rng.integers(0, 12))
        seed, fs = int(rng.integers(0, 1 << 30)), int(rng.integers(0, 100))
        io, ao, ro = Oracle(g.desc).render(g.camera, w, h, spp, depth, seed=seed, rng_mode=2, aux=True,
                                           first_sample=fs)
        ir, ar, rr = Reference(g.desc).render(g.camera, w, h, spp, depth, seed=seed, aux=True, first_sample=fs)
        assert io.tobytes() == ir.tobytes() and ao.tobytes() == ar.tobytes() and ro == rr, (kind, w, h, spp, depth)


def test_oracle_non_finite_geometry_matches_reference(built):
    """NaN and huge coordinates in triangles (flat and instanced) and
    spheres: the oracle builds the reference's trees (std::min / std::max
    decide where a NaN coordinate lands in a box) and returns the
    reference's hits and renders."""
    from oracle.oracle import Oracle, Reference, build_trees, ref_available, reference_trees
    if not ref_available():
        pytest.skip("reference harness absent")
    from handmade import non_finite_instances, non_finite_scene, non_finite_spheres
    d, rays = non_finite_scene(built)
    r = Reference(d.desc)
    mine, ref = build_trees(d.desc).arrays[0], reference_trees(r, d.desc).arrays[0]
    assert mine[0].tobytes() == ref[0].tobytes() and np.array_equal(mine[1], ref[1])
    o = Oracle(d.desc)
    hr, bad = r.trace_closest(rays)
    assert o.trace_closest(rays).tobytes() == hr.tobytes()
    assert np.array_equal(o.trace_any(rays), r.trace_any(rays))
    # instances of a mesh with NaN in triangle boxes: mesh bounds and instance
    # boxes as aabb::grow makes them
    g, rays = non_finite_instances(built)
    r = Reference(g.desc)
    for mine, ref in zip(build_trees(g.desc).arrays, reference_trees(r, g.desc).arrays):
        assert mine[0].tobytes() == ref[0].tobytes() and np.array_equal(mine[1], ref[1])
    o = Oracle(g.desc)
    assert o.trace_closest(rays).tobytes() == r.trace_closest(rays)[0].tobytes()
    assert np.array_equal(o.trace_any(rays), r.trace_any(rays))
    # spheres and a large sphere with NaN or huge centres and radii
    d, rays = non_finite_spheres(built)
    r = Reference(d.desc)
    mine, ref = build_trees(d.desc).arrays[0], reference_trees(r, d.desc).arrays[0]
    assert mine[0].tobytes() == ref[0].tobytes() and np.array_equal(mine[1], ref[1])
    o = Oracle(d.desc)
    assert o.trace_closest(rays).tobytes() == r.trace_closest(rays)[0].tobytes()
    assert np.array_equal(o.trace_any(rays), r.trace_any(rays))
    # whole renders through all three scenes: same images, guides and ray counts
    cam = built.camera_look_at((0.0, 0.5, 6.0), (0.0, 0.0, 0.0), 50.0, 1.5)
    for desc, c in ((non_finite_scene(built)[0].desc, cam), (non_finite_spheres(built)[0].desc, cam),
                    (g.desc, g.camera)):
        o, r = Oracle(desc), Reference(desc)
        io, ao, ro = o.render(c, 24, 16, 3, 10, seed=3, rng_mode=2, aux=True)
        ir, ar, rr = r.render(c, 24, 16, 3, 10, seed=3, aux=True)
        assert io.tobytes() == ir.tobytes() and ao.tobytes() == ar.tobytes() and ro == rr


def test_oracle_adversarial_rays_match_reference(built):
    """Rays with infinite, signed-zero, denormal and huge components: oracle
    = reference, closest and any hit. Rays with NaN components send the
    reference's walk round the root without end (it crashes); the oracle
    stops its walk at the stack bound instead, and must survive them."""
    from handmade import NAN_ORIGIN_RAY, adversarial_rays
    from oracle.oracle import Oracle, Reference, ref_available
    from photon_tracer_b200 import abi
    rays = adversarial_rays(9, 20000)
    for kind, param in ((abi.PT_GEN_ROOM_MESH, 3), (abi.PT_GEN_INSTANCES, 150), (abi.PT_GEN_REF_MATERIALS, 0)):
        g = built.Generated(kind, seed=2, param=param)
        o = Oracle(g.desc)
        o.trace_closest(np.concatenate([adversarial_rays(10, 2000, nan=True), NAN_ORIGIN_RAY]))
        if ref_available():
            r = Reference(g.desc)
            assert o.trace_closest(rays).tobytes() == r.trace_closest(rays)[0].tobytes()
            assert np.array_equal(o.trace_any(rays), r.trace_any(rays))


def test_oracle_material_renders_match_reference_fixture(built):
    """Renders the reference made of four random-material scenes (metal fuzz
    above 1 among them), pinned as a fixture: the oracle reproduces image,
    guides and ray count without the reference present."""
    from handmade import random_material_scene
    from oracle.oracle import Oracle
    f = golden("ref_material_renders.npz")
    for seed in range(4):
        d, cam = random_material_scene(built, 500 + seed)
        img, aux, rays = Oracle(d.desc).render(cam, 24, 16, 4, 10, seed=seed, rng_mode=2, aux=True)
        assert img.tobytes() == f[f"s{seed}_image"].tobytes() and aux.tobytes() == f[f"s{seed}_aux"].tobytes()
        assert rays == int(f[f"s{seed}_rays"])


def test_oracle_random_materials_match_reference(built):
    """Random scenes over all four material kinds and their edge parameters
    (metal fuzz above 1, dielectric ior at and below 1, negative radii,
    emitters): oracle renders equal the reference's, image, guides and ray
    count."""
    from handmade import random_material_scene
    from oracle.oracle import Oracle, Reference, ref_available
    if not ref_available():
        pytest.skip("reference harness absent")
    for seed in range(8):
        d, cam = random_material_scene(built, 500 + seed)
        o, r = Oracle(d.desc), Reference(d.desc)
        io, ao, ro = o.render(cam, 24, 16, 4, 10, seed=seed, rng_mode=2, aux=True)
        ir, ar, rr = r.render(cam, 24, 16, 4, 10, seed=seed, aux=True)
        assert io.tobytes() == ir.tobytes() and ao.tobytes() == ar.tobytes() and ro == rr, seed


def test_oracle_lights_and_sphere_radii_match_reference(built):
    """Next-event estimation over many (overlapping, tiny, huge) lights, and
    spheres of zero, negative-zero, denormal-scale and huge radius: oracle
    hits and renders equal the reference's."""
    from handmade import light_and_radius_scene
    from oracle.oracle import Oracle, Reference, ref_available
    if not ref_available():
        pytest.skip("reference harness absent")
    for seed in range(6):
        d, cam = light_and_radius_scene(built, 2100 + seed)
        o, r = Oracle(d.desc), Reference(d.desc)
        rays = built.generate_rays(seed, [-5, -5, -5], [5, 5, 5], 4000)
        assert o.trace_closest(rays).tobytes() == r.trace_closest(rays)[0].tobytes()
        io, ao, ro = o.render(cam, 24, 16, 4, 10, seed=seed, rng_mode=2, aux=True)
        ir, ar, rr = r.render(cam, 24, 16, 4, 10, seed=seed, aux=True)
        assert io.tobytes() == ir.tobytes() and ao.tobytes() == ar.tobytes() and ro == rr, seed


def test_camera_matches_reference_including_degenerate(built):
    """pt_camera_look_at at 16:9 against the reference's camera constructor:
    random placements and fields of view, and degenerate ones (eye at the
    target, looking straight up or down, fov 0 and 179.9, eye at 1e30)."""
    from oracle.oracle import ref_available, ref_camera
    if not ref_available():
        pytest.skip("reference harness absent")
    rng = np.random.default_rng(4)
    cases = [((0, 0, 0), (0, 0, 0), 40.0), ((0, 5, 0), (0, 0, 0), 40.0), ((0, -5, 0), (0, 0, 0), 40.0),
             ((1, 2, 3), (1, 2, 3.0001), 1e-3), ((1, 2, 3), (4, 5, 6), 179.9), ((1, 2, 3), (4, 5, 6), 0.0),
             ((1e30, 0, 0), (0, 0, 0), 40.0), ((0, 0, 1e-30), (0, 0, 0), 40.0)]
    cases += [(tuple(rng.normal(0, 10, 3)), tuple(rng.normal(0, 1, 3)), float(rng.uniform(1, 170))) for _ in range(200)]
    for lf, la, v in cases:
        assert bytes(memoryview(built.camera_look_at(lf, la, v))) == bytes(memoryview(ref_camera(lf, la, v))), (lf, la, v)


def test_triangle_init_matches_reference(built):
    """pt_triangle_init derives e1, e2 and the face normal from the corners
    bit for bit as the reference's triangle constructor does, over corners
    from 1e-3 to 1e3 in scale."""
    import ctypes as C
    from handmade import scene_from
    from oracle.oracle import Reference, ref_available
    from photon_tracer_b200 import abi
    if not ref_available():
        pytest.skip("reference harness absent")
    rng = np.random.default_rng(1)
    tris = [built.triangle(*(rng.normal(0, 10 ** rng.uniform(-3, 3), 3) for _ in range(3))) for _ in range(500)]
    d = scene_from(built, [abi.pt_material(type=0, albedo=abi.F3(0.5, 0.5, 0.5))], (), tris)
    r = Reference(d.desc)
    out = (C.c_float * 12)()
    for i, t in enumerate(tris):
        r.lib.ref_triangle_fields(r.h, -1, i, out)
        mine = np.array([list(t.p0), list(t.e1), list(t.e2), list(t.face_normal)], np.float32)
        assert mine.tobytes() == np.array(out[:], np.float32).tobytes(), i
        assert list(t.n0) == list(t.face_normal) == list(t.n2)


def test_instance_transforms_match_reference(built):
    """pt_affine_inverse gives the reference's affine::inverse bit for bit
    (singular matrices included: infinities and NaN alike), and with it the
    oracle traces and renders instances under random rotations, mirrors,
    flattening and a 1e-20 scale as the reference does."""
    import ctypes as C
    from handmade import random_transform_instances
    from oracle.oracle import Oracle, Reference, ref_available
    if not ref_available():
        pytest.skip("reference harness absent")
    out = (C.c_float * 12)()
    for singular in (True, False):
        g = random_transform_instances(built, 3, singular)
        d = g.desc
        r = Reference(d)
        for k in range(d.n_instances):
            r.lib.ref_instance_to_object(r.h, k, out)
            x = d.instances[k].to_object
            mine = [x.m[i][j] for i in range(3) for j in range(3)] + list(x.t)
            assert np.array(mine, np.float32).tobytes() == np.array(out[:], np.float32).tobytes(), k
    o = Oracle(d)
    rays = built.generate_rays(4, [-40, -1, -40], [40, 30, 40], 20000)
    assert o.trace_closest(rays).tobytes() == r.trace_closest(rays)[0].tobytes()
    assert np.array_equal(o.trace_any(rays), r.trace_any(rays))
    io, ao, ro = o.render(g.camera, 24, 16, 3, 10, seed=3, rng_mode=2, aux=True)
    ir, ar, rr = r.render(g.camera, 24, 16, 3, 10, seed=3, aux=True)
    assert io.tobytes() == ir.tobytes() and ao.tobytes() == ar.tobytes() and ro == rr


def test_oracle_edge_hits_match_reference_fixture(built):
    """Closest and any hits the reference made for adversarial rays (room
    scene) and on the NaN-geometry scenes, pinned as a fixture: the oracle
    reproduces them without the reference present."""
    from handmade import non_finite_scene, non_finite_spheres
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    f = golden("ref_edge_hits.npz")
    g = built.Generated(abi.PT_GEN_ROOM_MESH, seed=2, param=3)
    scenes = [("adversarial", g.desc), ("nan_triangles", non_finite_scene(built)[0].desc),
              ("nan_spheres", non_finite_spheres(built)[0].desc)]
    for name, desc in scenes:
        o = Oracle(desc)
        rays = f[f"{name}_rays"]
        assert o.trace_closest(rays).view(np.uint32).reshape(-1, 6).tobytes() == f[f"{name}_hits"].tobytes(), name
        assert np.array_equal(o.trace_any(rays), f[f"{name}_occluded"]), name


def test_oracle_denoise_matches_reference(built):
    """The oracle's a-trous filter against the reference's denoise: bit for
    bit on the committed fixture (a render of the reference's and random
    planes), and live on other random inputs when the reference is built."""
    from oracle.oracle import oracle_denoise, ref_available, ref_denoise
    f = golden("ref_denoise.npz")
    for name in ("render", "random"):
        got = oracle_denoise(f[f"{name}_color"], f[f"{name}_albedo"], f[f"{name}_normal"], f[f"{name}_variance"])
        assert got.tobytes() == f[f"{name}_out"].tobytes(), name
    if ref_available():
        rng = np.random.default_rng(3)
        for h, w in ((17, 29), (64, 5)):
            c, al = rng.random((h, w, 3), dtype=np.float32) * 4, rng.random((h, w, 3), dtype=np.float32)
            nrm, var = rng.normal(size=(h, w, 3)).astype(np.float32), rng.random((h, w), dtype=np.float32)
            assert oracle_denoise(c, al, nrm, var).tobytes() == ref_denoise(c, al, nrm, var).tobytes()


def test_sampler_known_answers(built):
    """The Sobol pairs (sampler.hpp) of the oracle against the reference's, and
    the superset-XOR form of the second Sobol dimension the GPU computes."""
    from oracle.oracle import oracle_sample_2d, ref_available, ref_sample_2d
    rng = np.random.default_rng(0)
    cases = [(int(rng.integers(0, 2**63)), int(rng.integers(0, 4000)), int(rng.integers(0, 3000)),
              int(rng.integers(0, 2**20)), int(b), int(po)) for b, po in [(-1, 0), (0, 0), (0, 1), (1, 0), (1, 1)]
             for _ in range(40)]
    if ref_available():
        for c in cases:
            assert np.array_equal(oracle_sample_2d(*c), ref_sample_2d(*c)), c

    def table_sobol(i):
        v = [1 << 31]
        for k in range(1, 32):
            v.append(v[-1] ^ (v[-1] >> 1))
        r = 0
        for k in range(32):
            if i >> k & 1:
                r ^= v[k]
        return int(f"{r:032b}"[::-1], 2)

    def superset_xor(r):
        r ^= (r >> 1) & 0x55555555
        r ^= (r >> 2) & 0x33333333
        r ^= (r >> 4) & 0x0F0F0F0F
        r ^= (r >> 8) & 0x00FF00FF
        r ^= (r >> 16) & 0x0000FFFF
        return r

    for i in [0, 1, 2, 3, 0xFFFFFFFF, 0x80000000] + [int(x) for x in rng.integers(0, 2**32, 2000)]:
        assert table_sobol(i) == superset_xor(i), hex(i)


def test_generators_match_reference_scenes(built):
    """materials / field / room built by the library equal the reference's make_scene / make_room_scene."""
    import ctypes as C
    from oracle.oracle import ref_available, ref_lib
    if not ref_available():
        pytest.skip("reference harness absent")
    from photon_tracer_b200 import abi
    for gen, sid in [(abi.PT_GEN_REF_MATERIALS, 0), (abi.PT_GEN_REF_FIELD, 1), (abi.PT_GEN_REF_ROOM, 3)]:
        g = built.Generated(gen)
        a = abi.desc_arrays(g.desc)
        counts = (C.c_uint32 * 4)()
        ref_lib().ref_builtin_scene(sid, counts, None, None)
        sph = np.zeros((counts[0], 4), np.float32)
        tri = np.zeros((counts[2], 9), np.float32)
        ref_lib().ref_builtin_scene(sid, counts, sph.ctypes.data_as(C.c_void_p), tri.ctypes.data_as(C.c_void_p))
        assert counts[0] == len(a["spheres"]) and counts[1] == len(a["large_spheres"]) and counts[2] == len(a["triangles"])
        mine_s = np.concatenate([a["spheres"]["center"], a["spheres"]["radius"][:, None]], axis=1)
        assert mine_s.tobytes() == sph.tobytes()
        mine_t = np.concatenate([a["triangles"]["p0"], a["triangles"]["e1"], a["triangles"]["e2"]], axis=1)
        assert mine_t.tobytes() == tri.tobytes()


def test_generated_fields_match_reference_constructors(built):
    """e1, e2, face normal (triangle ctor) and to_object (affine::inverse) as the reference computes them."""
    import ctypes as C
    from oracle.oracle import Reference, ref_available
    if not ref_available():
        pytest.skip("reference harness absent")
    from photon_tracer_b200 import abi
    g = built.Generated(abi.PT_GEN_INSTANCES, seed=3, param=200)
    r = Reference(g.desc)
    a = abi.desc_arrays(g.desc)
    out = np.zeros(12, np.float32)
    for m, tris in enumerate(a["meshes"]):
        for i in range(0, len(tris), max(1, len(tris) // 200)):
            r.lib.ref_triangle_fields(r.h, m, i, out.ctypes.data_as(C.c_void_p))
            mine = np.concatenate([tris[i]["p0"], tris[i]["e1"], tris[i]["e2"], tris[i]["face_normal"]])
            assert mine.tobytes() == out.tobytes()
    for k in range(len(a["instances"])):
        r.lib.ref_instance_to_object(r.h, k, out.ctypes.data_as(C.c_void_p))
        x = a["instances"][k]["to_object"]
        assert np.concatenate([x["m"].ravel(), x["t"]]).tobytes() == out.tobytes()


def block_z(image, mean, sigma, seeds, block=20, floor=2e-4):
    """render_test.py's check_scene statistics: worst |z| per block, per block
    row and per image channel against the fixture (tests/render_test.py:151-182)."""
    h, w, _ = image.shape
    bw, bh = w // block, h // block
    means = image[:bh * block, :bw * block].reshape(bh, block, bw, block, 3).mean(axis=(1, 3), dtype=np.float64)
    diffs = means.reshape(-1) - mean
    scale = np.sqrt(1 + 1 / seeds)
    var = (np.maximum(sigma, floor) * scale) ** 2
    worst_block = np.max(np.abs(diffs) / np.sqrt(var))
    d3, v3 = diffs.reshape(bh, bw, 3), var.reshape(bh, bw, 3)
    worst_row = np.max(np.abs(d3.sum(axis=1)) / np.sqrt(v3.sum(axis=1)))
    image_z = d3.sum(axis=(0, 1)) / np.sqrt(v3.sum(axis=(0, 1)))
    return worst_block, worst_row, np.max(np.abs(image_z))


def test_reference_fixture_is_reproduced_by_reference_on_generated_scene(built):
    """The reference, rendering the library's rebuild of its materials scene,
    passes its own statistical fixture (tests/reference.json thresholds)."""
    from oracle.oracle import Reference, ref_available
    if not ref_available():
        pytest.skip("reference harness absent")
    import json
    from photon_tracer_b200 import abi
    f = golden("reference_blocks.npz")
    meta = json.loads(str(f["meta"]))
    g = built.Generated(abi.PT_GEN_REF_MATERIALS)
    img, _, _ = Reference(g.desc).render(g.camera, meta["width"], meta["width"] * 9 // 16, meta["spp"], 10, seed=1,
                                        threads=os.cpu_count())
    b, r, i = block_z(img, f["materials_mean"], f["materials_sigma"], meta["seeds"])
    assert b <= 10 and r <= 6 and i <= 5, (b, r, i)
