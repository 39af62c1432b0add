"""Ray queries on the GPU through the C ABI, against the oracle: closest hits
(kind, primitive, sub-triangle, t, u, v) must be bit-identical, any-hit
answers identical, traversal work counters identical."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden
from handmade import NAN_ORIGIN_RAY, adversarial_rays
from handmade import non_finite_instances, non_finite_scene, non_finite_spheres
from handmade import scene_from as _scene_from, tri as _tri

pytestmark = pytest.mark.gpu

HIT_FIXTURES = sorted(f for f in os.listdir(GOLDEN) if f.startswith("ref_hits_"))


@pytest.fixture(scope="module")
def pt(built):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return built


def canonical(h):
    """Hit records as 6 words, with every NaN t/u/v replaced by one pattern:
    IEEE 754 leaves the payload of a NaN from an invalid operation (0/0) to
    the hardware (x86 gives 0xffc00000, the GPU 0x7fffffff), so only
    NaN-ness is compared."""
    w = h.view(np.uint32).reshape(-1, 6).copy()
    f = w[:, 3:].view(np.float32)
    w[:, 3:][np.isnan(f)] = 0x7FC00000
    return w


def assert_hits_equal(got, want, rays=None):
    if got.tobytes() == want.tobytes():
        return
    bad = np.nonzero(canonical(got) != canonical(want))[0]
    if len(bad) == 0:
        return
    i = int(bad[0])
    msg = f"{len(np.unique(bad))} rays differ; first ray {i}: got {got[i]} want {want[i]}"
    if rays is not None:
        msg += f" ray {rays[i]}"
    raise AssertionError(msg)


@pytest.mark.parametrize("name", HIT_FIXTURES)
def test_hits_match_reference_fixture(pt, name):
    f = golden(name)
    g = pt.Generated(int(f["kind"]), seed=1, param=int(f["param"]))
    s = pt.Scene(g)
    hits = s.trace_closest(f["rays"])
    assert_hits_equal(hits, f["hits"].reshape(-1).view(hits.dtype), f["rays"])
    assert np.array_equal(s.trace_any(f["rays"]), f["occluded"])


def test_room_mesh_ray_set_bit_exact(pt):
    """The 81,920-triangle room scene and the seeded ray-query set (origins in
    the room, directions uniform on the sphere): the first 1M rays against
    the oracle, bit for bit, and the traversal counters equal."""
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_ROOM_MESH, seed=1)
    s = pt.Scene(g)
    o = Oracle(g.desc)
    rays = pt.generate_rays(1, [-1, -1, -1], [1, 1, 1], 1 << 20)
    assert_hits_equal(s.trace_closest(rays), o.trace_closest(rays), rays)
    sub = rays[:200000]
    _, counts = o.trace_closest(sub, counts=True)
    assert np.array_equal(s.trace_count(sub), counts)
    occ_gpu = s.trace_any(rays, 0.001, 0.5)
    assert np.array_equal(occ_gpu, o.trace_any(rays, 0.001, 0.5))


def test_full_ray_set_bit_exact(pt):
    """All 16,777,216 rays of the query set (origins uniform in the room,
    directions uniform on the sphere, t in [0.001, 1000]): every GPU closest
    hit equals the oracle's bit for bit, every any-hit answer (t_max 0.5)
    too, and the set is deterministic. The oracle runs on all host cores."""
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_ROOM_MESH, seed=1)
    s = pt.Scene(g)
    rays = pt.generate_rays(1, [-1, -1, -1], [1, 1, 1], 1 << 24)
    h1 = s.trace_closest(rays)
    h2 = s.trace_closest(rays)
    assert h1.tobytes() == h2.tobytes()
    o = Oracle(g.desc)
    threads = os.cpu_count() or 1
    assert_hits_equal(h1, o.trace_closest(rays, threads=threads), rays)
    assert np.array_equal(s.trace_any(rays, 0.001, 0.5), o.trace_any(rays, 0.001, 0.5, threads=threads))
    # inside a closed room (open front) most rays hit something
    assert (h1["kind"] != abi.PT_HIT_NONE).mean() > 0.8


@pytest.mark.parametrize("kind,param,box", [
    ("RANDOM_SPHERES", 0, ([-12, 0, -12], [12, 3, 12])),
    ("INSTANCES", 0, ([-100, 0, -100], [100, 8, 100])),
    ("REF_FIELD", 0, ([-3, -0.5, -3], [3, 1.5, 0])),
    ("BATCH_SCENE", 0, ([-2, -2, -2], [2, 2, 2])),
])
def test_generators_bit_exact(pt, kind, param, box):
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    g = pt.Generated(getattr(abi, "PT_GEN_" + kind), seed=5, param=param)
    s = pt.Scene(g)
    o = Oracle(g.desc)
    rays = pt.generate_rays(11, box[0], box[1], 100000)
    assert_hits_equal(s.trace_closest(rays), o.trace_closest(rays), rays)
    assert np.array_equal(s.trace_any(rays), o.trace_any(rays))
    _, counts = o.trace_closest(rays[:20000], counts=True)
    assert np.array_equal(s.trace_count(rays[:20000]), counts)


def test_no_bvh_mode(pt):
    """geometry::build(false): every primitive tested in order (materials default)."""
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    for gen in (abi.PT_GEN_REF_MATERIALS, abi.PT_GEN_REF_FIELD):
        g = pt.Generated(gen, seed=1, use_bvh=0)
        s = pt.Scene(g)
        rays = pt.generate_rays(2, [-2, -0.5, -2], [2, 1, 0.5], 50000)
        assert_hits_equal(s.trace_closest(rays), Oracle(g.desc).trace_closest(rays), rays)


def test_edge_cases_ties_empty_degenerate(pt):
    """Equal-t ties (duplicate and coplanar triangles, concentric spheres),
    degenerate triangles, an empty scene, axis-aligned and zero directions."""
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    m = [abi.pt_material(type=0, albedo=abi.F3(0.5, 0.5, 0.5))]
    tris = []
    for k in range(12):  # a stack of duplicates at z = 0 and z = -1, plus slivers
        tris.append(_tri(pt, (-1, -1, 0), (1, -1, 0), (0, 1, 0)))
        tris.append(_tri(pt, (-1, -1, -1), (1, -1, -1), (1, 1, -1)))
    tris.append(_tri(pt, (0, 0, 0.5), (1, 0, 0.5), (2, 0, 0.5)))  # zero area
    sph = [abi.pt_sphere(center=abi.F3(0, 0, -2), radius=0.5), abi.pt_sphere(center=abi.F3(0, 0, -2), radius=0.5),
           abi.pt_sphere(center=abi.F3(0, 0, -2), radius=-0.3)]
    lg = [abi.pt_sphere(center=abi.F3(0, -1001, 0), radius=1000.0)]
    rng = np.random.default_rng(3)
    rays = np.concatenate([
        np.concatenate([rng.uniform(-1, 1, (3000, 2)), np.full((3000, 1), 3), rng.normal(0, 0.2, (3000, 2)),
                        np.full((3000, 1), -1)], axis=1),
        np.array([[0, 0, 3, 0, 0, -1], [0.2, -0.3, 3, 0, 0, -1], [0, 0, 3, 0, 0, 0], [0, 0, 0, 1, 0, 0],
                  [0.5, 0, 0.5, -1, 0, 0], [0, 5, -2, 0, -1, 0], [0, 0, 3, 0, 0, -0.0]]),
    ]).astype(np.float32)
    for use_bvh in (1, 0):
        d = _scene_from(pt, m, sph, tris, lg, use_bvh)
        s = pt.Scene(d.desc_ptr)
        o = Oracle(d.desc)
        assert_hits_equal(s.trace_closest(rays), o.trace_closest(rays), rays)
        assert np.array_equal(s.trace_any(rays), o.trace_any(rays))
    empty = _scene_from(pt, m)
    s = pt.Scene(empty.desc_ptr)
    h = s.trace_closest(rays)
    assert np.all(h["kind"] == abi.PT_HIT_NONE) and not s.trace_any(rays).any()


def test_non_finite_geometry(pt):
    """Triangles with a NaN or huge vertex among ordinary ones: node boxes
    that hold NaN turn the fast slab test off for the whole scene (the
    NaN-ignoring min / max and the near-plane choice are exact only for
    ordered boxes), so hits stay those of the reference's SSE arithmetic
    (the oracle's agreement with the reference on this scene is checked in
    tests/test_oracle.py)."""
    from oracle.oracle import Oracle
    d, rays = non_finite_scene(pt)
    s = pt.Scene(d.desc_ptr)
    o = Oracle(d.desc)
    assert_hits_equal(s.trace_closest(rays), o.trace_closest(rays), rays)
    assert np.array_equal(s.trace_any(rays), o.trace_any(rays))
    g, rays = non_finite_instances(pt)
    s = pt.Scene(g)
    o = Oracle(g.desc)
    assert_hits_equal(s.trace_closest(rays), o.trace_closest(rays), rays)
    assert np.array_equal(s.trace_any(rays), o.trace_any(rays))
    d, rays = non_finite_spheres(pt)
    s = pt.Scene(d.desc_ptr)
    o = Oracle(d.desc)
    assert_hits_equal(s.trace_closest(rays), o.trace_closest(rays), rays)
    assert np.array_equal(s.trace_any(rays), o.trace_any(rays))


def test_adversarial_rays(pt):
    """Rays with infinite, signed-zero, denormal and huge components match
    the oracle bit for bit (which matches the reference on them,
    tests/test_oracle.py). A ray with a NaN origin, on which the reference's
    walk never ends, makes the call fail with PT_ERR_STACK_OVERFLOW (the
    stack bound is checked on every push), and the scene stays usable."""
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    rays = adversarial_rays(9, 20000)
    for kind, param in ((abi.PT_GEN_ROOM_MESH, 3), (abi.PT_GEN_INSTANCES, 150), (abi.PT_GEN_REF_MATERIALS, 0)):
        g = pt.Generated(kind, seed=2, param=param)
        s = pt.Scene(g)
        o = Oracle(g.desc)
        assert_hits_equal(s.trace_closest(rays), o.trace_closest(rays), rays)
        assert np.array_equal(s.trace_any(rays), o.trace_any(rays))
    g = pt.Generated(abi.PT_GEN_ROOM_MESH, seed=2, param=3)
    s = pt.Scene(g)
    with pytest.raises(abi.PhotonError) as e:
        s.trace_closest(NAN_ORIGIN_RAY)
    assert e.value.status == abi.PT_ERR_STACK_OVERFLOW
    assert_hits_equal(s.trace_closest(rays), Oracle(g.desc).trace_closest(rays), rays)


def test_device_buffers_entry_point(pt):
    """pt_trace_closest_device on torch tensors equals the host-buffer call."""
    import torch
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_ROOM_MESH, seed=1, param=4)
    s = pt.Scene(g)
    rays = pt.generate_rays(9, [-1, -1, -1], [1, 1, 1], 65536)
    d_rays = torch.from_numpy(rays).cuda()
    d_hits = torch.empty((len(rays), 6), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    s.trace_closest_device(d_rays.data_ptr(), len(rays), d_hits.data_ptr(), stream=stream)
    s.sync(stream)
    got = d_hits.cpu().numpy().view(abi.HIT_DTYPE).reshape(-1)
    assert_hits_equal(got, s.trace_closest(rays), rays)


@pytest.mark.parametrize("scene_id", [0, 1, 3])
def test_geometry_bridge_on_reference_scenes(pt, scene_id):
    """The reference's own scenes, built by its build_world and handed over
    through include/photon_cuda_geometry.hpp with the reference's own trees:
    GPU closest-hit t equals geometry::hit's rec.t on every ray, and the
    rendered frame's mean agrees with render_row_linear's."""
    import json
    import subprocess
    from conftest import ROOT
    shim = os.path.join(ROOT, "oracle", "_ref", "shim_check")
    if not os.path.exists(shim):
        pytest.skip("the bridge check binary was not built (needs the reference checkout at build time)")
    res = subprocess.run([shim, str(scene_id)], capture_output=True, text=True, timeout=600)
    out = json.loads(res.stdout)
    assert res.returncode == 0 and out["hit_mismatch"] == 0, out
    assert abs(out["gpu_mean"] - out["cpu_mean"]) <= 0.02 * out["cpu_mean"], out
    assert abs(out["gpu_rays"] - out["cpu_rays"]) <= 0.02 * out["cpu_rays"], out


def test_l2_read_probe(pt):
    """pt_measure_l2_read: the L2 read rate the traversal roofline is reported
    against -- a positive, finite rate, and refusals of bad arguments."""
    import ctypes as C
    from photon_tracer_b200 import abi
    lib = pt.load()
    gbs = C.c_double()
    assert lib.pt_measure_l2_read(8 << 20, 8, C.byref(gbs)) == abi.PT_OK, lib.pt_last_error()
    assert 100.0 < gbs.value < 1e6
    assert lib.pt_measure_l2_read(16, 8, C.byref(gbs)) == abi.PT_ERR_INVALID_ARG
    assert lib.pt_measure_l2_read(8 << 20, 0, C.byref(gbs)) == abi.PT_ERR_INVALID_ARG
