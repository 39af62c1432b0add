"""The library's host BVH builder produces exactly the reference's bvh::build
trees (nodes and leaf order), so hit ties resolve identically. Checked
against the reference itself where oracle/_ref exists, and against the
committed digests of the reference's trees everywhere. CPU only."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN


def digest(trees):
    out = []
    for t in trees.arrays:
        if t is None:
            out.append(None)
        else:
            out.append([int(len(t[0])), int(len(t[1])), hashlib.sha256(t[0].tobytes() + t[1].tobytes()).hexdigest()])
    return out


def test_trees_match_reference_digests(built):
    from oracle.oracle import build_trees
    cases = json.load(open(os.path.join(GOLDEN, "ref_trees.json")))
    for name, c in cases.items():
        g = built.Generated(c["kind"], seed=1, param=c["param"])
        assert digest(build_trees(g.desc)) == c["trees"], name


def test_trees_match_reference_live(built):
    from oracle.oracle import Reference, build_trees, ref_available, reference_trees
    if not ref_available():
        pytest.skip("reference harness absent")
    from photon_tracer_b200 import abi
    for kind, param, seed in [(abi.PT_GEN_ROOM_MESH, 4, 3), (abi.PT_GEN_RANDOM_SPHERES, 1500, 9),
                              (abi.PT_GEN_INSTANCES, 500, 2), (abi.PT_GEN_BATCH_SCENE, 0, 17)]:
        g = built.Generated(kind, seed=seed, param=param)
        assert digest(build_trees(g.desc)) == digest(reference_trees(Reference(g.desc), g.desc))


@pytest.mark.parametrize("n", [0, 1, 2, 3, 8, 9, 17, 1000])
def test_builder_invariants(built, n):
    rng = np.random.default_rng(n)
    lo = rng.uniform(-10, 10, (n, 3)).astype(np.float32)
    boxes = np.concatenate([lo, lo + rng.uniform(0, 1, (n, 3)).astype(np.float32)], axis=1)
    nodes, order = built.bvh_build(boxes)
    assert sorted(order.tolist()) == list(range(n))
    if n == 0:
        assert len(nodes) == 0
        return
    # every primitive appears in exactly one leaf; children boxes contain their primitives
    seen = np.zeros(n, int)
    for nd in nodes:
        for c in range(4):
            cnt, first = nd["count"][c], nd["first"][c]
            if cnt:
                idx = order[first:first + cnt]
                seen[idx] += 1
                assert np.all(boxes[idx, :3] >= nd["lo"][:, c] - 0) and np.all(boxes[idx, 3:] <= nd["hi"][:, c])
                assert cnt <= 8 or n == 1
            elif np.isfinite(nd["lo"][0][c]):
                assert first < len(nodes)
    assert np.all(seen == 1)


def test_builder_coincident_and_flat_boxes(built):
    """All centroids in one point: no SAH split exists and the node halves."""
    boxes = np.tile(np.array([[0, 0, 0, 1, 1, 1]], np.float32), (40, 1))
    nodes, order = built.bvh_build(boxes)
    assert sorted(order.tolist()) == list(range(40))
    flat = np.array([[i, 0, 0, i + 0.5, 0, 0] for i in range(20)], np.float32)  # zero-area boxes
    nodes, order = built.bvh_build(flat)
    assert sorted(order.tolist()) == list(range(20))


def test_builder_matches_reference_on_mesh_boxes(built):
    """Mesh trees of random triangle soups, built by both."""
    from oracle.oracle import Reference, ref_available, reference_trees, triangle_boxes
    if not ref_available():
        pytest.skip("reference harness absent")
    import ctypes as C
    from photon_tracer_b200 import abi
    rng = np.random.default_rng(5)
    n = 3000
    tris = np.zeros(n, abi.TRIANGLE_DTYPE)
    p0 = rng.normal(0, 3, (n, 3)).astype(np.float32)
    p1 = (p0 + rng.normal(0, 0.3, (n, 3))).astype(np.float32)
    p2 = (p0 + rng.normal(0, 0.3, (n, 3))).astype(np.float32)
    tris["p0"], tris["p1"], tris["p2"] = p0, p1, p2
    tris["e1"], tris["e2"] = p1 - p0, p2 - p0
    mats = (abi.pt_material * 1)(abi.pt_material(type=0, albedo=abi.F3(0.5, 0.5, 0.5)))
    mesh = (abi.pt_mesh * 1)()
    mesh[0].triangles = C.cast(tris.ctypes.data, C.POINTER(abi.pt_triangle))
    mesh[0].n_triangles = n
    d = abi.pt_scene_desc(materials=mats, n_materials=1, meshes=mesh, n_meshes=1, use_bvh=1, sky=1)
    ref_nodes, ref_order = reference_trees(Reference(d), d).arrays[2]
    nodes, order = built.bvh_build(triangle_boxes(tris))
    assert nodes.tobytes() == ref_nodes.tobytes()
    assert np.array_equal(order, ref_order)
