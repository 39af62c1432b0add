"""The GPU BVH builder (pt_bvh_build_gpu) against the host builder
(pt_bvh_build, itself checked node for node against the reference's
bvh::build in tests/test_bvh_build.py): identical nodes and leaf order, byte
for byte, on random, degenerate and signed-zero inputs of every size class
(single primitives, subtrees handled by one thread, level-parallel nodes)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pt(built):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return built


def random_boxes(rng, n, spread=10.0, size=0.05):
    c = rng.random((n, 3)) * spread
    e = rng.random((n, 3)) * size
    return np.concatenate([c - e, c + e], 1).astype(np.float32)


def assert_same(pt, boxes):
    nh, oh = pt.bvh_build(boxes)
    ng, og = pt.bvh_build(boxes, gpu=True)
    assert len(ng) == len(nh)
    np.testing.assert_array_equal(og, oh)
    assert ng.tobytes() == nh.tobytes()


@pytest.mark.parametrize("n", [1, 2, 3, 8, 9, 100, 128, 129, 1000, 4097, 70000])
def test_random_boxes(pt, n):
    assert_same(pt, random_boxes(np.random.default_rng(n), n))


def test_large_random(pt):
    rng = np.random.default_rng(7)
    boxes = random_boxes(rng, 400000, spread=100.0, size=0.2)
    t = time.perf_counter()
    nh, oh = pt.bvh_build(boxes)
    t_host = time.perf_counter() - t
    pt.bvh_build(boxes[:1000], gpu=True)  # warm
    t = time.perf_counter()
    ng, og = pt.bvh_build(boxes, gpu=True)
    t_gpu = time.perf_counter() - t
    print(f"400k boxes: host {t_host * 1e3:.1f} ms, gpu {t_gpu * 1e3:.1f} ms")
    np.testing.assert_array_equal(og, oh)
    assert ng.tobytes() == nh.tobytes()


def test_clustered_and_degenerate(pt):
    rng = np.random.default_rng(3)
    # identical boxes: no centroid extent, median splits only
    same = np.tile(np.array([[0, 0, 0, 1, 1, 1]], np.float32), (3000, 1))
    assert_same(pt, same)
    # centroids on a line, and in a few tight clusters
    line = np.zeros((5000, 6), np.float32)
    line[:, 0] = rng.random(5000)
    line[:, 3] = line[:, 0] + 0.01
    line[:, 4:6] = 0.01
    assert_same(pt, line)
    centers = rng.random((5, 3)) * 10
    cl = centers[rng.integers(0, 5, 20000)] + rng.normal(0, 1e-3, (20000, 3))
    assert_same(pt, np.concatenate([cl - 0.01, cl + 0.01], 1).astype(np.float32))


def test_signed_zeros(pt):
    """-0.0 and +0.0 compare equal but are different bytes: the box of a node
    keeps the first one met in primitive order, as std::min / std::max do."""
    rng = np.random.default_rng(11)
    n = 30000
    b = random_boxes(rng, n, spread=2.0, size=0.5) - 1.0
    zero = rng.random((n, 6)) < 0.3
    sign = np.where(rng.random((n, 6)) < 0.5, -1.0, 1.0).astype(np.float32)
    b = np.where(zero, np.float32(0.0) * sign, b).astype(np.float32)
    b[:, 3:] = np.maximum(b[:, 3:], b[:, :3])
    assert_same(pt, b)


def test_mesh_triangles(pt):
    """Triangle boxes of the displaced icosphere (the room scene's mesh, 81,920
    triangles), in the generator's order."""
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_ROOM_MESH, seed=1)
    d = g.desc
    tris = np.ctypeslib.as_array(d.triangles, (d.n_triangles,))
    p0, p1, p2 = tris["p0"], tris["p1"], tris["p2"]
    boxes = np.concatenate([np.minimum(np.minimum(p0, p1), p2) - 1e-4, np.maximum(np.maximum(p0, p1), p2) + 1e-4],
                           1).astype(np.float32)
    assert_same(pt, boxes)
