"""Scene descriptions stored as compact fixtures (tests/golden/ref_scene_*.npz)
and rebuilt as pt_scene_desc, for the reference's OBJ scenes (the teapot, the
crowd, the spot crowd), which need the reference's model files to build.

A fixture keeps what the reference's scene holds: materials, spheres, large
spheres, instances as they are, and each triangle list as a table of unique
corners (position, vertex normal, texture coordinates) with three corner
numbers and a material per triangle. The derived triangle fields (edges, face
normal) are recomputed in float32 in the order of the reference's triangle
constructor (include/triangle.hpp:32-35), which gives its bytes back.
"""
import ctypes as C

import numpy as np

CORNER = 8  # floats per unique corner: position 3, normal 3, uv 2


def _corners(tris):
    """(table of unique corners, corner numbers per triangle) of a triangle array."""
    rows = np.concatenate([np.concatenate([tris[p], tris[n], tris["uv"][:, 2 * k:2 * k + 2]], axis=1)
                           for k, (p, n) in enumerate((("p0", "n0"), ("p1", "n1"), ("p2", "n2")))])
    rows = np.ascontiguousarray(rows, np.float32)
    keys = rows.view(np.dtype((np.void, 4 * CORNER))).reshape(-1)
    _, first, inverse = np.unique(keys, return_index=True, return_inverse=True)
    # table in order of first use, so the file does not depend on the sort order of the bytes
    order = np.argsort(first)
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    table = rows[first[order]]
    idx = rank[inverse.reshape(-1)].reshape(3, -1).T.astype(np.uint32)
    return table, np.ascontiguousarray(idx)


def _cross(a, b):
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1], a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1).astype(np.float32)


def _normalize(v):
    """vec3::normalize (include/vec3.hpp:95-98): each component over
    sqrt(x*x + y*y + z*z), in float32."""
    v = v.astype(np.float32)
    with np.errstate(all="ignore"):
        length = np.sqrt((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2], dtype=np.float32)
        return (v / length[:, None]).astype(np.float32)


def make_triangles(p0, p1, p2, n0, n1, n2, material, uv):
    """pt_triangle rows as the reference's smooth constructor makes them:
    e1 = p1 - p0, e2 = p2 - p0, face normal = cross(e1, e2).normalize()."""
    from photon_tracer_b200 import abi
    out = np.zeros(len(p0), abi.TRIANGLE_DTYPE)
    out["p0"], out["p1"], out["p2"] = p0, p1, p2
    out["n0"], out["n1"], out["n2"] = n0, n1, n2
    out["e1"] = (p1 - p0).astype(np.float32)
    out["e2"] = (p2 - p0).astype(np.float32)
    out["face_normal"] = _normalize(_cross(out["e1"], out["e2"]))
    out["material"] = material
    out["uv"] = uv
    return out


def _triangles_from(table, idx, material):
    c = [table[idx[:, k]] for k in range(3)]
    uv = np.concatenate([x[:, 6:8] for x in c], axis=1)
    return make_triangles(c[0][:, 0:3], c[1][:, 0:3], c[2][:, 0:3], c[0][:, 3:6], c[1][:, 3:6], c[2][:, 3:6],
                          material, uv)


def pack(desc, camera) -> dict:
    """The arrays of a fixture for a description and its camera."""
    from photon_tracer_b200 import abi
    a = abi.desc_arrays(desc)
    out = {"materials": a["materials"].copy(), "spheres": a["spheres"].copy(),
           "large_spheres": a["large_spheres"].copy(), "instances": a["instances"].copy(),
           "flags": np.array([desc.sky, desc.sample_lights, desc.use_bvh], np.int32),
           "camera": np.frombuffer(bytes(camera), np.float32).copy(), "n_meshes": np.int32(len(a["meshes"]))}
    for name, tris in [("flat", a["triangles"])] + [(f"mesh{m}", t) for m, t in enumerate(a["meshes"])]:
        table, idx = _corners(tris)
        out[f"{name}_corners"], out[f"{name}_index"] = table, idx
        out[f"{name}_material"] = tris["material"].copy()
    for k in range(desc.n_textures):
        t = desc.textures[k]
        out[f"texture{k}"] = np.ctypeslib.as_array(t.rgb, (t.height, t.width, 3)).copy()
    return out


def triangles_of(f, name):
    return _triangles_from(f[f"{name}_corners"], f[f"{name}_index"], f[f"{name}_material"])


def flatten_instances(f):
    """make_crowd_scene with flatten (include/renderer.hpp:316-325): every
    instance's copy of its mesh written out as world-space triangles -- corners
    by to_world.point, vertex normals by to_object.transposed(n).normalize(),
    the instance's material unless it has none -- in float32 and the
    reference's order of operations. Returns the flat triangle array."""
    from photon_tracer_b200 import abi
    meshes = [triangles_of(f, f"mesh{m}") for m in range(int(f["n_meshes"]))]
    out = []
    for inst in f["instances"]:
        t = meshes[int(inst["mesh"])]
        m, tt = inst["to_world"]["m"].astype(np.float32), inst["to_world"]["t"].astype(np.float32)
        mi = inst["to_object"]["m"].astype(np.float32)

        def point(p):  # affine::point: ((m0 x + m1 y) + m2 z) + t per row
            return np.stack([((m[r, 0] * p[:, 0] + m[r, 1] * p[:, 1]) + m[r, 2] * p[:, 2]) + tt[r]
                             for r in range(3)], axis=1).astype(np.float32)

        def normal(n):  # affine::transposed with to_object, then normalize
            return _normalize(np.stack([(mi[0, c] * n[:, 0] + mi[1, c] * n[:, 1]) + mi[2, c] * n[:, 2]
                                        for c in range(3)], axis=1))

        mat = t["material"] if inst["material"] == abi.PT_NO_MATERIAL else np.full(len(t), inst["material"], np.uint32)
        out.append(make_triangles(point(t["p0"]), point(t["p1"]), point(t["p2"]), normal(t["n0"]), normal(t["n1"]),
                                  normal(t["n2"]), mat, t["uv"]))
    return np.concatenate(out)


class FixtureScene:
    """A pt_scene_desc rebuilt from a fixture (trees left to the library's
    builder, which makes the reference's trees), kept alive with its arrays.
    flatten: the instances written out as flat triangles instead."""

    def __init__(self, f, flatten: bool = False):
        from photon_tracer_b200 import abi
        self.materials = np.ascontiguousarray(f["materials"])
        self.spheres = np.ascontiguousarray(f["spheres"])
        self.large = np.ascontiguousarray(f["large_spheres"])
        flat = triangles_of(f, "flat")
        if flatten:
            flat = np.concatenate([flat, flatten_instances(f)])
            self.instances = np.zeros(0, abi.INSTANCE_DTYPE)
            self.mesh_tris = []
        else:
            self.instances = np.ascontiguousarray(f["instances"])
            self.mesh_tris = [triangles_of(f, f"mesh{m}") for m in range(int(f["n_meshes"]))]
        self.triangles = np.ascontiguousarray(flat)
        self.meshes = (abi.pt_mesh * max(1, len(self.mesh_tris)))()
        for m, t in enumerate(self.mesh_tris):
            self.meshes[m].triangles = C.cast(t.ctypes.data, C.POINTER(abi.pt_triangle))
            self.meshes[m].n_triangles = len(t)
        names = sorted(k for k in f.files if k.startswith("texture"))
        self.texture_pixels = [np.ascontiguousarray(f[k], np.uint8) for k in names]
        self.textures = (abi.pt_texture * max(1, len(names)))()
        for k, px in enumerate(self.texture_pixels):
            self.textures[k].width, self.textures[k].height = px.shape[1], px.shape[0]
            self.textures[k].rgb = px.ctypes.data_as(C.POINTER(C.c_uint8))
        sky, sample_lights, use_bvh = (int(x) for x in f["flags"])

        def ptr(a, t):
            return C.cast(a.ctypes.data, C.POINTER(t)) if len(a) else None
        self.desc = abi.pt_scene_desc(
            materials=ptr(self.materials, abi.pt_material), n_materials=len(self.materials),
            spheres=ptr(self.spheres, abi.pt_sphere), n_spheres=len(self.spheres),
            large_spheres=ptr(self.large, abi.pt_sphere), n_large_spheres=len(self.large),
            triangles=ptr(self.triangles, abi.pt_triangle), n_triangles=len(self.triangles),
            meshes=self.meshes if self.mesh_tris else None, n_meshes=len(self.mesh_tris),
            instances=ptr(self.instances, abi.pt_instance), n_instances=len(self.instances),
            sky=sky, sample_lights=sample_lights, use_bvh=use_bvh,
            textures=self.textures if names else None, n_textures=len(names))
        self.desc_ptr = C.pointer(self.desc)
        self.camera = abi.pt_camera.from_buffer_copy(np.ascontiguousarray(f["camera"], np.float32).tobytes())
