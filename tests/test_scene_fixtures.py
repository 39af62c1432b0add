"""The reference's OBJ scenes (teapot, crowd, spot crowd) kept as fixtures
(tests/scene_fixture.py): the descriptions rebuilt from them give the trees
the reference's geometry::build made, the flattened crowd equals the
reference's own flattening, and the oracle renders them as the reference
does. The GPU checks of these scenes are in tests/test_gpu_render.py."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import golden

SCENES = ["teapot", "crowd", "spot_crowd"]
MODELS = {"teapot": (2, "models/teapot.obj", 20, 0.0), "crowd": (4, "models/teapot.obj", 8, 0.0),
          "spot_crowd": (4, "models/spot/spot.obj", 6, 150.0)}


def digest(t):
    nodes, order = t
    return [int(len(nodes)), int(len(order)),
            hashlib.sha256(nodes.tobytes() + np.asarray(order, np.uint32).tobytes()).hexdigest()]


@pytest.mark.parametrize("name", SCENES)
def test_rebuilt_scene_gives_the_reference_trees(built, name):
    from oracle.oracle import build_trees
    from scene_fixture import FixtureScene
    f = golden(f"ref_scene_{name}.npz")
    want = json.loads(str(f["trees"]))
    d = FixtureScene(f)
    trees = build_trees(d.desc)
    got = {"flat": digest(trees.arrays[0]), "instances": digest(trees.arrays[1])}
    got.update({f"mesh{m}": digest(t) for m, t in enumerate(trees.arrays[2:])})
    assert got == want


def reference_model(name):
    from oracle.build import REFERENCE
    from oracle.oracle import ref_available
    path = os.path.join(REFERENCE, MODELS[name][1])
    if not ref_available() or not os.path.exists(path):
        pytest.skip("reference checkout or harness absent")
    return path


def test_flattened_crowd_equals_the_references(built):
    """make_crowd_scene(flatten) of the reference against the fixture's
    instances written out in tests/scene_fixture.py: every triangle field
    bit for bit, materials by value."""
    from oracle.oracle import RefWorld
    from photon_tracer_b200 import abi
    from scene_fixture import flatten_instances
    path = reference_model("crowd")
    f = golden("ref_scene_crowd.npz")
    w = RefWorld(4, path, 8, True)
    ref = abi.desc_arrays(w.desc)
    mine = flatten_instances(f)
    for k in abi.TRIANGLE_DTYPE.names:
        if k != "material":
            assert mine[k].tobytes() == ref["triangles"][k].tobytes(), k
    assert f["materials"][mine["material"]].tobytes() == ref["materials"][ref["triangles"]["material"]].tobytes()


@pytest.mark.parametrize("name", SCENES)
def test_fixture_equals_the_references_scene(built, name):
    from oracle.oracle import RefWorld
    from photon_tracer_b200 import abi
    from scene_fixture import FixtureScene
    sid, _, side, turn = MODELS[name]
    w = RefWorld(sid, reference_model(name), side, False, turn)
    d = FixtureScene(golden(f"ref_scene_{name}.npz"))
    a, b = abi.desc_arrays(w.desc), abi.desc_arrays(d.desc)
    for k in ("materials", "spheres", "large_spheres", "triangles", "instances"):
        assert a[k].tobytes() == b[k].tobytes(), k
    assert [m.tobytes() for m in a["meshes"]] == [m.tobytes() for m in b["meshes"]]
    assert bytes(w.camera) == bytes(d.camera)


@pytest.mark.parametrize("name,flatten", [("teapot", False), ("crowd", False), ("crowd", True), ("spot_crowd", False)])
def test_oracle_renders_fixture_scenes_like_reference(built, name, flatten):
    from oracle.oracle import Oracle, Reference, ref_available
    from scene_fixture import FixtureScene
    if not ref_available():
        pytest.skip("reference harness absent")
    d = FixtureScene(golden(f"ref_scene_{name}.npz"), flatten=flatten)
    o, r = Oracle(d.desc), Reference(d.desc)
    io, ao, ro = o.render(d.camera, 32, 18, 2, 10, seed=3, rng_mode=2, aux=True)
    ir, ar, rr = r.render(d.camera, 32, 18, 2, 10, seed=3, aux=True)
    assert io.tobytes() == ir.tobytes() and ao.tobytes() == ar.tobytes() and ro == rr


def test_material_fixture_states_replay_in_the_oracle(built):
    """The captured per-sample states of the material fixture drive the
    oracle's snapshot mode to the reference's images exactly (so the GPU test
    that replays them checks the GPU, not the capture)."""
    from handmade import random_material_scene
    from oracle.oracle import Oracle
    f = golden("ref_material_renders.npz")
    for seed in range(4):
        d, cam = random_material_scene(built, 500 + seed)
        img, aux, rays = Oracle(d.desc).render(cam, 24, 16, 4, 10, seed=seed, rng_mode=1, states=f[f"s{seed}_states"],
                                               aux=True)
        assert img.tobytes() == f[f"s{seed}_image"].tobytes() and aux.tobytes() == f[f"s{seed}_aux"].tobytes()
        assert rays == int(f[f"s{seed}_rays"])
