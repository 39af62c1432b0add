"""Hand-made scene descriptions for the traversal tests (no GPU needed to
build them)."""
import ctypes as C

import numpy as np


def scene_from(pt, materials, spheres=(), tris=(), large=(), use_bvh=1):
    """A small hand-made description (kept alive on the returned object)."""
    from photon_tracer_b200 import abi

    class Desc:
        pass
    d = Desc()
    d.mats = (abi.pt_material * max(1, len(materials)))(*materials)
    d.sph = (abi.pt_sphere * max(1, len(spheres)))(*spheres)
    d.lg = (abi.pt_sphere * max(1, len(large)))(*large)
    d.tri = (abi.pt_triangle * max(1, len(tris)))(*tris)
    d.desc = abi.pt_scene_desc(materials=d.mats, n_materials=len(materials), spheres=d.sph, n_spheres=len(spheres),
                               large_spheres=d.lg, n_large_spheres=len(large), triangles=d.tri, n_triangles=len(tris),
                               use_bvh=use_bvh, sky=1, sample_lights=1)
    d.desc_ptr = C.pointer(d.desc)
    return d


def tri(pt, a, b, c, mat=0):
    from photon_tracer_b200 import abi
    a, b, c = (np.array(x, np.float32) for x in (a, b, c))
    e1, e2 = b - a, c - a
    n = np.cross(e1.astype(np.float64), e2.astype(np.float64))
    n = (n / np.linalg.norm(n)).astype(np.float32)
    t = abi.pt_triangle(material=mat)
    for name, v in [("p0", a), ("e1", e1), ("e2", e2), ("n0", n), ("n1", n), ("n2", n), ("face_normal", n),
                    ("p1", b), ("p2", c)]:
        setattr(t, name, abi.F3(*v.tolist()))
    return t


def set_corners(t, a, b, c):
    """Corners a, b, c with the edges and face normal the reference's
    triangle constructor derives from them (float32, its evaluation order:
    e = corner - p0, face normal = cross(e1, e2) / its length per component)."""
    from photon_tracer_b200 import abi
    p0, p1, p2 = (np.array(x, np.float32) for x in (a, b, c))
    e1, e2 = p1 - p0, p2 - p0
    n = np.array([e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]],
                 np.float32)
    with np.errstate(all="ignore"):
        length = np.sqrt(np.float32(n[0] * n[0] + n[1] * n[1]) + n[2] * n[2], dtype=np.float32)
        n = (n / length).astype(np.float32)
    for name, v in (("p0", p0), ("p1", p1), ("p2", p2), ("e1", e1), ("e2", e2), ("face_normal", n)):
        setattr(t, name, abi.F3(*v.tolist()))


def non_finite_scene(pt):
    """200 random triangles plus three with a NaN or a -1e30 coordinate, and
    20,000 random rays through them: (description, rays)."""
    from photon_tracer_b200 import abi
    m = [abi.pt_material(type=0, albedo=abi.F3(0.5, 0.5, 0.5))]
    rng = np.random.default_rng(21)
    tris = []
    for k in range(200):
        c = rng.uniform(-2, 2, 3)
        t = tri(pt, (0, 0, 0), (1, 0, 0), (0, 1, 0))
        set_corners(t, c, c + rng.uniform(-0.3, 0.3, 3), c + rng.uniform(-0.3, 0.3, 3))
        tris.append(t)
    nan = float("nan")
    bad = [((nan, 0, 0), (1, 0, 0), (0, 1, 0)), ((0, 0, 0.2), (nan, nan, 0.2), (0, 1, 0.2)),
           ((-1e30, 0, -0.5), (1, 0, -0.5), (0, 1, -0.5))]
    for a, b, c in bad:
        t = tri(pt, (0, 0, 0), (1, 0, 0), (0, 1, 0))
        set_corners(t, a, b, c)
        tris.insert(int(rng.integers(len(tris))), t)
    d = scene_from(pt, m, (), tris)
    rays = np.concatenate([rng.uniform(-3, 3, (20000, 3)), rng.normal(0, 1, (20000, 3))], 1).astype(np.float32)
    return d, rays


def non_finite_instances(pt):
    """The 150-instance scene with NaN first corners in two triangles of a
    mesh and a -1e30 corner in a third (edges and face normals recomputed
    to match), and
    20,000 random rays: (generated scene, rays). A NaN first corner makes the
    triangle's box hold NaN, which the mesh bounds and the instance boxes
    then skip or carry the way aabb::grow does."""
    from photon_tracer_b200 import abi
    g = pt.Generated(abi.PT_GEN_INSTANCES, seed=4, param=150)
    mt = g.desc.meshes[0].triangles
    for k in (3, 40, 7):
        p0, p1, p2 = (list(getattr(mt[k], n)) for n in ("p0", "p1", "p2"))
        if k == 7:
            p2[1] = -1e30
        else:
            p0[0] = float("nan")
        set_corners(mt[k], p0, p1, p2)
    rays = pt.generate_rays(4, [-40, -1, -40], [40, 30, 40], 20000)
    return g, rays


def non_finite_spheres(pt):
    """100 random spheres with a NaN centre, a NaN radius and a 1e30 centre
    among them, a ground sphere and a NaN-centred large sphere, and 20,000
    random rays: (description, rays)."""
    from photon_tracer_b200 import abi
    m = [abi.pt_material(type=0, albedo=abi.F3(0.5, 0.5, 0.5))]
    rng = np.random.default_rng(5)
    sph = [abi.pt_sphere(center=abi.F3(*rng.uniform(-2, 2, 3).tolist()), radius=float(rng.uniform(0.1, 0.4)))
           for _ in range(100)]
    nan = float("nan")
    sph[10] = abi.pt_sphere(center=abi.F3(nan, 0, 0), radius=0.3)
    sph[50] = abi.pt_sphere(center=abi.F3(0, 0, 0), radius=nan)
    sph[70] = abi.pt_sphere(center=abi.F3(0.5, 1e30, 0), radius=0.2)
    large = [abi.pt_sphere(center=abi.F3(0, -1001, 0), radius=1000.0),
             abi.pt_sphere(center=abi.F3(nan, 0, 0), radius=1000.0)]
    d = scene_from(pt, m, sph, [tri(pt, (0, 0, 0), (1, 0, 0), (0, 1, 0))], large)
    rays = np.concatenate([rng.uniform(-3, 3, (20000, 3)), rng.normal(0, 1, (20000, 3))], 1).astype(np.float32)
    return d, rays


def adversarial_rays(seed, n, nan=False):
    """Random rays in [-3, 3]^6 with 15% of their components replaced by
    infinities, signed zeros, denormals or +-1e38 (and NaN when nan=True)."""
    rng = np.random.default_rng(seed)
    vals = [np.inf, -np.inf, 0.0, -0.0, 1e-45, -1e-45, 1e38, -1e38, 1.0, -1.0, 0.5] + ([np.nan] if nan else [])
    vals = np.array(vals, np.float32)
    rays = rng.uniform(-3, 3, (n, 6)).astype(np.float32)
    mask = rng.random((n, 6)) < 0.15
    rays[mask] = vals[rng.integers(len(vals), size=int(mask.sum()))]
    return rays


# A ray with a NaN origin: every slab test passes, empty child slots (first 0)
# re-enter the root, and the walk never ends; the reference overruns its
# stack on it.
NAN_ORIGIN_RAY = np.array([[-1.636903, np.nan, np.nan, 0.6391732, -0.9654722, 2.588736]], np.float32)


def random_material_scene(pt, seed):
    """Eight random materials of all four kinds (metal fuzz up to 1.7, which
    the reference clamps to 1; dielectric ior 0.7 to 2.4), 20 spheres (some
    with a negative radius), 30 triangles and a ground sphere, and a camera:
    (description, camera)."""
    from photon_tracer_b200 import abi
    rng = np.random.default_rng(seed)
    mats = []
    for k in range(8):
        t = int(rng.integers(4))
        mats.append(abi.pt_material(type=t, albedo=abi.F3(*rng.uniform(0, 1, 3).tolist()),
                                    emission=abi.F3(*(rng.uniform(0, 4, 3) if t == 3 else np.zeros(3)).tolist()),
                                    fuzz=float(rng.choice([0.0, 0.3, 1.0, 1.7])),
                                    ior=float(rng.choice([1.0, 1.5, 0.7, 2.4]))))
    sph = [abi.pt_sphere(center=abi.F3(*rng.uniform(-2, 2, 3).tolist()), radius=float(rng.choice([0.3, 0.6, -0.4])),
                         material=int(rng.integers(8))) for _ in range(20)]
    tris = []
    for _ in range(30):
        c = rng.uniform(-2, 2, 3)
        t = tri(pt, (0, 0, 0), (1, 0, 0), (0, 1, 0), mat=int(rng.integers(8)))
        set_corners(t, c, c + rng.uniform(-0.8, 0.8, 3), c + rng.uniform(-0.8, 0.8, 3))
        tris.append(t)
    large = [abi.pt_sphere(center=abi.F3(0, -1001, 0), radius=1000.0, material=int(rng.integers(8)))]
    cam = pt.camera_look_at(tuple(rng.uniform(-5, 5, 3).tolist()), (0.0, 0.0, 0.0), 40.0, 1.5)
    return scene_from(pt, mats, sph, tris, large), cam


def random_transform_instances(pt, seed, singular=False):
    """The 60-instance scene with every to_world replaced by a random rotation
    times per-axis scales from {0.5, 1, 2, -1, 1e-3} (mirrors and flattening
    included; instance 9 scaled by 1e-20; with singular=True instance 5's
    last row zeroed) and to_object from pt.affine_inverse: the generated
    scene."""
    from photon_tracer_b200 import abi
    rng = np.random.default_rng(seed)
    g = pt.Generated(abi.PT_GEN_INSTANCES, seed=4, param=60)
    d = g.desc
    for k in range(d.n_instances):
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        m = (q * rng.choice([0.5, 1.0, 2.0, -1.0, 1e-3], 3)).astype(np.float32)
        if k == 9:
            m = np.eye(3, dtype=np.float32) * np.float32(1e-20)
        if singular and k == 5:
            m[2] = 0
        t = rng.uniform(-30, 30, 3).astype(np.float32)
        inst = d.instances[k]
        for r in range(3):
            for c in range(3):
                inst.to_world.m[r][c] = float(m[r, c])
            inst.to_world.t[r] = float(t[r])
        inst.to_object = pt.affine_inverse(inst.to_world)
    return g


def light_and_radius_scene(pt, seed):
    """Many emissive spheres (some overlapping, tiny or huge), spheres of
    radius 0, -0, 1e-30, 1e-7, +-0.5 and 1e15 over all four material kinds,
    two large spheres of 1e2..1e5 radius, and a camera: (description, camera)."""
    from photon_tracer_b200 import abi
    rng = np.random.default_rng(seed)
    mats = [abi.pt_material(type=0, albedo=abi.F3(*rng.uniform(0, 1, 3).tolist())),
            abi.pt_material(type=3, emission=abi.F3(*rng.uniform(0.5, 8, 3).tolist())),
            abi.pt_material(type=1, albedo=abi.F3(0.8, 0.8, 0.8), fuzz=0.2),
            abi.pt_material(type=2, ior=1.5)]
    sph = [abi.pt_sphere(center=abi.F3(*rng.uniform(-3, 3, 3).tolist()), radius=float(rng.uniform(0.05, 1.5)),
                         material=1) for _ in range(int(rng.integers(1, 12)))]
    radii = [0.0, -0.0, 1e-30, 1e-7, 0.5, -0.5, 1e15, 1.0]
    sph += [abi.pt_sphere(center=abi.F3(*rng.uniform(-3, 3, 3).tolist()), radius=float(rng.choice(radii)),
                          material=int(rng.integers(4))) for _ in range(15)]
    large = [abi.pt_sphere(center=abi.F3(*(rng.uniform(-1, 1, 3) * 10 ** rng.uniform(2, 5)).tolist()),
                           radius=float(10 ** rng.uniform(2, 5)), material=int(rng.choice([0, 2]))) for _ in range(2)]
    cam = pt.camera_look_at(tuple(rng.uniform(-6, 6, 3).tolist()), (0.0, 0.0, 0.0), float(rng.uniform(20, 90)), 1.5)
    return scene_from(pt, mats, sph, (), large), cam
