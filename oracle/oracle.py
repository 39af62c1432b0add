"""TEST INFRASTRUCTURE: Python access to the two CPU checkers.

* Oracle    -- the plain-C restatement (oracle/pt_oracle.c -> libptoracle.so).
* Reference -- the reference itself (oracle/ref_harness.cpp -> _ref/libptref.so),
               present where the reference checkout was available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product (photon_tracer_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from photon_tracer_b200 import abi
from photon_tracer_b200.api import bvh_build

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "libptoracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libptref.so")

P = C.c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


_olib = None
_rlib = None


def oracle_lib() -> C.CDLL:
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            from oracle import build as _b
            _b.build_oracle()
        _olib = C.CDLL(ORACLE_LIB)
        L = _olib
        L.po_scene_create.restype = P
        L.po_scene_create.argtypes = [C.POINTER(abi.pt_scene_desc), C.POINTER(abi.pt_bvh), C.POINTER(abi.pt_bvh),
                                      C.POINTER(abi.pt_bvh)]
        L.po_scene_destroy.argtypes = [P]
        L.po_trace_closest.argtypes = [P, P, C.c_size_t, C.c_float, C.c_float, P, P]
        L.po_trace_any.argtypes = [P, P, C.c_size_t, C.c_float, C.c_float, P]
        L.po_render.argtypes = [P, C.POINTER(abi.pt_camera), C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int,
                                C.c_int, P, C.c_int, C.c_int, P, P, C.POINTER(C.c_uint64), P]
        L.po_sample_2d.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_uint32, C.c_int, C.c_int, P]
        L.po_sample_stream_seed.restype = C.c_uint64
        L.po_sample_stream_seed.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_uint32]
        L.po_denoise.argtypes = [C.c_int, C.c_int, P, P, P, P, P]
        L.po_render_flags.argtypes = L.po_render.argtypes + [C.c_int]
        L.po_metal_lobe_pdf.restype = C.c_float
        L.po_metal_lobe_pdf.argtypes = [abi.F3, C.c_float, abi.F3]
    return _olib


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib() -> C.CDLL:
    global _rlib
    if _rlib is None:
        if not os.path.exists(REF_LIB):
            raise RuntimeError("oracle/_ref/libptref.so is absent (built from the reference checkout)")
        L = C.CDLL(REF_LIB)
        L.ref_scene_create.restype = P
        L.ref_scene_create.argtypes = [C.POINTER(abi.pt_scene_desc)]
        L.ref_scene_destroy.argtypes = [P]
        L.ref_triangle_fields.argtypes = [P, C.c_int, C.c_uint32, P]
        L.ref_instance_to_object.argtypes = [P, C.c_uint32, P]
        L.ref_tree.restype = C.c_uint32
        L.ref_tree.argtypes = [P, C.c_int, C.c_int, P, C.c_uint32, P, C.c_uint32, C.POINTER(C.c_uint32)]
        L.ref_trace_closest.argtypes = [P, P, C.c_size_t, C.c_float, C.c_float, P, C.POINTER(C.c_uint64)]
        L.ref_trace_any.argtypes = [P, P, C.c_size_t, C.c_float, C.c_float, P]
        L.ref_render.restype = C.c_uint64
        L.ref_render.argtypes = [P, C.POINTER(abi.pt_camera), C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int,
                                 C.c_int, C.c_int, P, P, C.c_int]
        L.ref_render_snapshot.restype = C.c_uint64
        L.ref_render_snapshot.argtypes = [P, C.POINTER(abi.pt_camera), C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64,
                                          C.c_int, C.c_int, C.c_int, P, P, P]
        L.ref_denoise.argtypes = [C.c_int, C.c_int, P, P, P, P, P, C.c_int]
        L.ref_sample_2d.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_uint32, C.c_int, C.c_int, P]
        L.ref_camera.argtypes = [abi.F3, abi.F3, C.c_double, C.POINTER(abi.pt_camera)]
        L.ref_camera_roundtrip.restype = C.c_int
        L.ref_camera_roundtrip.argtypes = [C.POINTER(abi.pt_camera)]
        L.ref_builtin_scene.argtypes = [C.c_int, C.POINTER(C.c_uint32), P, P]
        L.ref_write_image.restype = C.c_int
        L.ref_write_image.argtypes = [C.c_char_p, C.c_int, C.c_int, P]
        L.ref_world_create.restype = P
        L.ref_world_create.argtypes = [C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_double]
        L.ref_world_desc.restype = C.POINTER(abi.pt_scene_desc)
        L.ref_world_desc.argtypes = [P]
        L.ref_world_camera.restype = C.POINTER(abi.pt_camera)
        L.ref_world_camera.argtypes = [P]
        L.ref_world_destroy.argtypes = [P]
        _rlib = L
    return _rlib


# ---- the boxes geometry::build gives the builder (include/geometry.hpp:74-104) -------------
def triangle_boxes(tris: np.ndarray) -> np.ndarray:
    """triangle::bounding_box (include/triangle.hpp:76-83) in float32, with
    std::min / std::max over {p0, p1, p2}: the first element unless a later
    one compares less (greater), which also decides where a NaN coordinate
    survives (numpy's min / max would propagate every NaN)."""
    p0, p1, p2 = (np.asarray(tris[k], np.float32) for k in ("p0", "p1", "p2"))
    pad = np.float32(1e-4)
    lo, hi = p0.copy(), p0.copy()
    for p in (p1, p2):
        lo = np.where(p < lo, p, lo)
        hi = np.where(hi < p, p, hi)
    return np.concatenate([lo - pad, hi + pad], axis=1).astype(np.float32)


def sphere_boxes(sph: np.ndarray) -> np.ndarray:
    r = np.abs(sph["radius"]).astype(np.float32)[:, None]
    c = sph["center"].astype(np.float32)
    return np.concatenate([c - r, c + r], axis=1)


def affine_box(m: np.ndarray, t: np.ndarray, box: np.ndarray) -> np.ndarray:
    """affine::box (include/transform.hpp:62-70) in float32, reference order."""
    m = m.astype(np.float32)
    t = t.astype(np.float32)
    lo = np.full(3, np.inf, np.float32)
    hi = np.full(3, -np.inf, np.float32)
    for k in range(8):
        c = np.array([box[3] if k & 1 else box[0], box[4] if k & 2 else box[1], box[5] if k & 4 else box[2]],
                     np.float32)
        p = np.empty(3, np.float32)
        for r in range(3):
            v = np.float32(np.float32(m[r, 0] * c[0]) + np.float32(m[r, 1] * c[1]))
            v = np.float32(v + np.float32(m[r, 2] * c[2]))
            p[r] = np.float32(v + t[r])
        lo = np.where(p < lo, p, lo)  # aabb::grow: std::min / std::max (include/aabb.hpp:15-20)
        hi = np.where(hi < p, p, hi)
    return np.concatenate([lo, hi])


def _grow(vals: np.ndarray, lower: bool) -> np.float32:
    """aabb::grow folded over vals in order, from +inf (lower) or -inf: the
    first occurrence of the least (greatest) value that is not NaN, since a
    NaN never compares less (greater) than the running value."""
    v = np.asarray(vals, np.float32)
    ok = ~np.isnan(v)
    if not ok.any():
        return np.float32(np.inf if lower else -np.inf)
    best = v[ok].min() if lower else v[ok].max()
    return v[np.nonzero(ok & (v == best))[0][0]]


class Trees:
    """The BVHs of a scene (flat, instances, each mesh) as pt_bvh structs, with
    their arrays kept alive."""

    def __init__(self, flat, inst, meshes):
        self.arrays = [flat, inst] + list(meshes)
        self.flat = self._bvh(flat)
        self.inst = self._bvh(inst)
        self.meshes = (abi.pt_bvh * max(1, len(meshes)))()
        for i, m in enumerate(meshes):
            self.meshes[i] = self._bvh(m)

    @staticmethod
    def _bvh(t):
        b = abi.pt_bvh()
        if t is None:
            return b
        nodes, order = t
        b.nodes = C.cast(nodes.ctypes.data, C.POINTER(abi.pt_bvh_node)) if len(nodes) else None
        b.n_nodes = len(nodes)
        b.order = C.cast(order.ctypes.data, C.POINTER(C.c_uint32)) if len(order) else None
        b.n_order = len(order)
        return b


def build_trees(desc: abi.pt_scene_desc) -> Trees:
    """The trees geometry::build makes, with the library's builder."""
    a = abi.desc_arrays(desc)
    meshes, bounds = [], []
    for tris in a["meshes"]:
        boxes = triangle_boxes(tris)
        meshes.append(bvh_build(boxes))
        bounds.append(np.array([_grow(boxes[:, a], True) for a in range(3)] +
                               [_grow(boxes[:, 3 + a], False) for a in range(3)], np.float32) if len(boxes) else None)
    flat = inst = None
    if desc.use_bvh:
        boxes = np.concatenate([sphere_boxes(a["spheres"]), triangle_boxes(a["triangles"])]) \
            if len(a["triangles"]) else sphere_boxes(a["spheres"])
        flat = bvh_build(boxes.reshape(-1, 6))
        ib = np.array([affine_box(i["to_world"]["m"], i["to_world"]["t"], bounds[i["mesh"]]) for i in a["instances"]],
                      np.float32).reshape(-1, 6)
        inst = bvh_build(ib)
    return Trees(flat, inst, meshes)


def reference_trees(ref: "Reference", desc: abi.pt_scene_desc) -> Trees:
    """The trees the reference's geometry::build made."""
    def get(which, mesh=0):
        n_order = C.c_uint32()
        nn = ref.lib.ref_tree(ref.h, which, mesh, None, 0, None, 0, C.byref(n_order))
        nodes = np.zeros(nn, abi.NODE_DTYPE)
        order = np.zeros(n_order.value, np.uint32)
        ref.lib.ref_tree(ref.h, which, mesh, _ptr(nodes), nn, _ptr(order), n_order.value, C.byref(n_order))
        return nodes, order
    meshes = [get(2, m) for m in range(desc.n_meshes)]
    flat = get(0) if desc.use_bvh else None
    inst = get(1) if desc.use_bvh else None
    return Trees(flat, inst, meshes)


class Oracle:
    """The C restatement over one scene."""

    def __init__(self, desc: abi.pt_scene_desc, trees: Optional[Trees] = None):
        self.lib = oracle_lib()
        self.desc = desc
        self.trees = trees or build_trees(desc)
        self.h = self.lib.po_scene_create(C.byref(desc), C.byref(self.trees.flat), C.byref(self.trees.inst),
                                          self.trees.meshes)

    def close(self):
        if self.h:
            self.lib.po_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _chunks(n, threads):
        """Contiguous [a, b) ranges for `threads` workers (ctypes calls release
        the GIL, and the oracle's ray queries only read the scene)."""
        step = max(1, -(-n // max(1, threads)))
        return [(a, min(n, a + step)) for a in range(0, n, step)]

    def trace_closest(self, rays, tmin=0.001, tmax=1000.0, counts=False, threads=1):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.empty(len(rays), abi.HIT_DTYPE)
        c = np.zeros(5, np.uint64)
        if threads > 1 and not counts and len(rays) > threads:
            from concurrent.futures import ThreadPoolExecutor
            with ThreadPoolExecutor(threads) as ex:
                list(ex.map(lambda ab: self.lib.po_trace_closest(self.h, _ptr(rays[ab[0]:ab[1]]), ab[1] - ab[0], tmin,
                                                                 tmax, _ptr(out[ab[0]:ab[1]]), None),
                            self._chunks(len(rays), threads)))
            return out
        self.lib.po_trace_closest(self.h, _ptr(rays), len(rays), tmin, tmax, _ptr(out), _ptr(c) if counts else None)
        return (out, c) if counts else out

    def trace_any(self, rays, tmin=0.001, tmax=1000.0, threads=1):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.empty(len(rays), np.uint8)
        if threads > 1 and len(rays) > threads:
            from concurrent.futures import ThreadPoolExecutor
            with ThreadPoolExecutor(threads) as ex:
                list(ex.map(lambda ab: self.lib.po_trace_any(self.h, _ptr(rays[ab[0]:ab[1]]), ab[1] - ab[0], tmin, tmax,
                                                             _ptr(out[ab[0]:ab[1]])),
                            self._chunks(len(rays), threads)))
            return out
        self.lib.po_trace_any(self.h, _ptr(rays), len(rays), tmin, tmax, _ptr(out))
        return out

    def render(self, cam, width, height, spp, depth=10, seed=1, first_sample=0, rng_mode=0, states=None,
               row0=0, rows=None, aux=False, counts=False, flags=0):
        """rng_mode 0: per-sample streams, 1: snapshot states, 2: the reference's per-row stream.
        flags: PT_FLAG_* (PT_FLAG_NEE_EXTENDED: the extended light sampling)."""
        rows = height - row0 if rows is None else rows
        out = np.zeros((height, width, 3), np.float32)
        ax = np.zeros((height, width, 7), np.float32) if aux else None
        rays = C.c_uint64()
        c = np.zeros(5, np.uint64)
        st = None if states is None else np.ascontiguousarray(states, np.uint64)
        self.lib.po_render_flags(self.h, C.byref(cam), width, height, spp, depth, seed, first_sample, rng_mode,
                                 _ptr(st), row0, rows, _ptr(out), _ptr(ax), C.byref(rays), _ptr(c) if counts else None,
                                 flags)
        res = (out, ax, rays.value)
        return res + (c,) if counts else res


def sample_stream_seed(seed, i, j, s):
    return oracle_lib().po_sample_stream_seed(seed, i, j, s)


def oracle_sample_2d(seed, i, j, index, bounce, pair_offset):
    out = np.zeros(2, np.float32)
    oracle_lib().po_sample_2d(seed, i, j, index, bounce, pair_offset, _ptr(out))
    return out


def oracle_denoise(color, albedo, normal, variance):
    h, w = color.shape[:2]
    arrs = [np.ascontiguousarray(a, np.float32) for a in (color, albedo, normal, variance)]
    out = np.empty((h, w, 3), np.float32)
    oracle_lib().po_denoise(w, h, *[_ptr(a) for a in arrs], _ptr(out))
    return out


class Reference:
    """The reference's own geometry for a description (oracle/_ref)."""

    def __init__(self, desc: abi.pt_scene_desc):
        self.lib = ref_lib()
        self.desc = desc
        self.h = self.lib.ref_scene_create(C.byref(desc))

    def close(self):
        if self.h:
            self.lib.ref_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def trace_closest(self, rays, tmin=0.001, tmax=1000.0):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.empty(len(rays), abi.HIT_DTYPE)
        bad = C.c_uint64()
        self.lib.ref_trace_closest(self.h, _ptr(rays), len(rays), tmin, tmax, _ptr(out), C.byref(bad))
        return out, bad.value

    def trace_any(self, rays, tmin=0.001, tmax=1000.0):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.empty(len(rays), np.uint8)
        self.lib.ref_trace_any(self.h, _ptr(rays), len(rays), tmin, tmax, _ptr(out))
        return out

    def render(self, cam, width, height, spp, depth=10, seed=1, first_sample=0, row0=0, rows=None, aux=False,
               threads=1):
        rows = height - row0 if rows is None else rows
        out = np.zeros((height, width, 3), np.float32)
        ax = np.zeros((height, width, 7), np.float32) if aux else None
        rays = self.lib.ref_render(self.h, C.byref(cam), width, height, spp, depth, seed, first_sample, row0, rows,
                                   _ptr(out), _ptr(ax), threads)
        return out, ax, rays

    def render_snapshot(self, cam, width, height, spp, depth=10, seed=1, first_sample=0, row0=0, rows=None):
        """The reference's per-row stream with the state before each sample's
        path captured: (image, aux, rays, states[rows*W*spp, 4])."""
        rows = height - row0 if rows is None else rows
        out = np.zeros((height, width, 3), np.float32)
        ax = np.zeros((height, width, 7), np.float32)
        states = np.zeros((rows * width * spp, 4), np.uint64)
        rays = self.lib.ref_render_snapshot(self.h, C.byref(cam), width, height, spp, depth, seed, first_sample, row0,
                                            rows, _ptr(out), _ptr(ax), _ptr(states))
        return out, ax, rays, states


def ref_sample_2d(seed, i, j, index, bounce, pair_offset):
    out = np.zeros(2, np.float32)
    ref_lib().ref_sample_2d(seed, i, j, index, bounce, pair_offset, _ptr(out))
    return out


def ref_denoise(color, albedo, normal, variance, threads=1):
    h, w = color.shape[:2]
    arrs = [np.ascontiguousarray(a, np.float32) for a in (color, albedo, normal, variance)]
    out = np.empty((h, w, 3), np.float32)
    ref_lib().ref_denoise(w, h, *[_ptr(a) for a in arrs], _ptr(out), threads)
    return out


def ref_camera(lookfrom, lookat, vfov):
    cam = abi.pt_camera()
    ref_lib().ref_camera(abi.f3(lookfrom), abi.f3(lookat), vfov, C.byref(cam))
    return cam


class RefWorld:
    """One of the reference's own worlds as its CLI builds it (build_world in
    include/renderer.hpp:335-343, src/main.cpp:63-108): scene id 0 materials,
    1 field, 2 mesh (the OBJ between two spheres), 3 room, 4 crowd (side x
    side copies of the OBJ, flattened or instanced), with NEE on. desc points
    into the reference's geometry (trees included); camera is make_camera(id)."""

    MATERIALS, FIELD, MESH, ROOM, CROWD = 0, 1, 2, 3, 4

    def __init__(self, scene_id: int, obj_path: str = "", crowd_side: int = 20, flatten: bool = False,
                 turn_deg: float = 0.0):
        self.lib = ref_lib()
        self.h = self.lib.ref_world_create(scene_id, obj_path.encode(), crowd_side, int(flatten), turn_deg)
        self.desc = self.lib.ref_world_desc(self.h).contents
        self.camera = abi.pt_camera.from_buffer_copy(self.lib.ref_world_camera(self.h).contents)

    def close(self):
        if self.h:
            self.lib.ref_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def oracle_metal_lobe_pdf(mirror, fuzz, w):
    """The oracle's density of metal's scattered direction at unit direction w."""
    return float(oracle_lib().po_metal_lobe_pdf(abi.f3(mirror), float(fuzz), abi.f3(w)))
