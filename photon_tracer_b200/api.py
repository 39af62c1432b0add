"""Python host API over the C ABI: scenes, cameras, renders and ray queries.

It mirrors the reference's interface for the render path -- geometry /
camera / render_row_linear (photon_tracer include/renderer.hpp:411-416) --
with the work done by libphoton_cuda.so on the GPU. Host arrays are numpy;
device arrays are anything with a CUDA pointer (torch tensors here).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import abi
from .abi import check, f3, load


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---- cameras -------------------------------------------------------------------
def camera_look_at(lookfrom, lookat, vfov_deg: float, aspect: float = 16.0 / 9.0) -> abi.pt_camera:
    """camera(lookfrom, lookat, vfov) (include/camera.hpp:18-34) with an aspect ratio."""
    cam = abi.pt_camera()
    check(load().pt_camera_look_at(f3(lookfrom), f3(lookat), float(vfov_deg), float(aspect), C.byref(cam)))
    return cam


# ---- generated scenes ----------------------------------------------------------------
class Generated:
    """A procedural scene built by the library (pt_generate); owns its arrays."""

    def __init__(self, kind: int, seed: int = 1, param: int = 0, use_bvh: int = -1):
        lib = load()
        self.params = abi.pt_gen_params(kind=kind, param=param, seed=seed, use_bvh=use_bvh)
        h = C.c_void_p()
        check(lib.pt_generate(C.byref(self.params), C.byref(h)))
        self._h = h
        self.desc = lib.pt_generated_desc(h).contents
        self.camera = abi.pt_camera.from_buffer_copy(lib.pt_generated_camera(h).contents)
        self.width, self.height, self.spp = self.params.width, self.params.height, self.params.spp

    @property
    def desc_ptr(self):
        return load().pt_generated_desc(self._h)

    def close(self):
        if self._h:
            load().pt_generated_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generate_rays(seed: int, lo, hi, n: int) -> np.ndarray:
    """n rays (n x 6 float32): origins uniform in [lo, hi], directions uniform on the sphere."""
    out = np.empty((n, 6), np.float32)
    check(load().pt_generate_rays(seed, f3(lo), f3(hi), n, _ptr(out)))
    return out


# ---- BVH --------------------------------------------------------------------------
def triangle(p0, p1, p2, normals=None, material: int = 0, uv=None) -> "abi.pt_triangle":
    """A pt_triangle as the reference's constructors make it from its corners
    (e1, e2, face normal derived; normals = three vertex normals or None for a
    flat triangle); uv: six texture coordinates or None."""
    fl = lambda v, n: (C.c_float * n)(*[float(x) for x in np.asarray(v, np.float32).reshape(-1)])
    out = abi.pt_triangle()
    nrm = fl(normals, 9) if normals is not None else None
    check(load().pt_triangle_init(fl(p0, 3), fl(p1, 3), fl(p2, 3), nrm, int(material), C.byref(out)))
    if uv is not None:
        for k, x in enumerate(np.asarray(uv, np.float32).reshape(6)):
            out.uv[k] = float(x)
    return out


def affine_inverse(to_world: "abi.pt_affine") -> "abi.pt_affine":
    """The to_object an instance must carry for to_world (affine::inverse)."""
    out = abi.pt_affine()
    check(load().pt_affine_inverse(C.byref(to_world), C.byref(out)))
    return out


def bvh_build(boxes: np.ndarray, gpu: bool = False):
    """The library's builder (same nodes and order as the reference's bvh::build).
    boxes: (n, 6) float32 min xyz, max xyz. Returns (nodes structured array, order).
    gpu: build on the GPU (pt_bvh_build_gpu), the same result."""
    boxes = np.ascontiguousarray(boxes, np.float32)
    lib = load()
    nodes_p = C.POINTER(abi.pt_bvh_node)()
    order_p = C.POINTER(C.c_uint32)()
    nn = C.c_uint32()
    fn = lib.pt_bvh_build_gpu if gpu else lib.pt_bvh_build
    check(fn(_ptr(boxes), boxes.shape[0], C.byref(nodes_p), C.byref(nn), C.byref(order_p)))
    try:
        nodes = np.ctypeslib.as_array(C.cast(nodes_p, C.POINTER(C.c_uint8)), (nn.value * 128,)).copy()
        nodes = nodes.view(abi.NODE_DTYPE) if nn.value else np.zeros(0, abi.NODE_DTYPE)
        n = boxes.shape[0]
        order = np.ctypeslib.as_array(order_p, (n,)).copy() if n else np.zeros(0, np.uint32)
    finally:
        lib.pt_free(C.cast(nodes_p, C.c_void_p))
        lib.pt_free(C.cast(order_p, C.c_void_p))
    return nodes, order


# ---- scenes ---------------------------------------------------------------------------
@dataclass
class SceneInfo:
    n_nodes: int
    n_slots: int
    max_depth: int
    stack_entries: int
    device_bytes: int


class Scene:
    """A scene on the device (pt_scene_create): the repacked node arena."""

    def __init__(self, desc):
        """desc: a pt_scene_desc, a pointer to one, or a Generated / Geometry."""
        if hasattr(desc, "desc_ptr"):
            self._keep = desc
            desc = desc.desc_ptr
        elif isinstance(desc, abi.pt_scene_desc):
            desc = C.pointer(desc)
        h = C.c_void_p()
        check(load().pt_scene_create(desc, C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def info(self) -> SceneInfo:
        i = abi.pt_scene_info()
        check(load().pt_scene_get_info(self._h, C.byref(i)))
        return SceneInfo(i.n_nodes, i.n_slots, i.max_depth, i.stack_entries, i.device_bytes)

    def close(self):
        if getattr(self, "_h", None):
            load().pt_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- rendering --
    def render(self, cam, width: int, height: int, spp: int, max_bounces: int = 10, seed: int = 1,
               first_sample: int = 0, mode: int = abi.PT_MODE_AUTO, rng: int = abi.PT_RNG_SAMPLE,
               states: Optional[np.ndarray] = None, aux: bool = False, flags: int = 0):
        """A frame with host buffers. Returns (image H x W x 3 top row first, aux H x W x 7 or None, rays).
        flags: PT_FLAG_* (PT_FLAG_NEE_EXTENDED: light sampling toward emissive triangles and from rough metal)."""
        st = self.settings(width, height, spp, max_bounces, seed, first_sample, mode, rng, states, flags=flags)
        out = np.empty((height, width, 3), np.float32)
        ax = np.empty((height, width, 7), np.float32) if aux else None
        rays = C.c_uint64()
        check(load().pt_render(self._h, C.byref(cam), C.byref(st), _ptr(out), _ptr(ax), C.byref(rays)))
        return out, ax, rays.value

    @staticmethod
    def settings(width, height, spp, max_bounces=10, seed=1, first_sample=0, mode=abi.PT_MODE_AUTO,
                 rng=abi.PT_RNG_SAMPLE, states=None, states_ptr=None, flags=0) -> abi.pt_settings:
        st = abi.pt_settings(width=width, height=height, spp=spp, max_bounces=max_bounces, seed=seed,
                             first_sample=first_sample, mode=mode, rng=rng, flags=flags)
        if states is not None:
            states = np.ascontiguousarray(states, np.uint64)
            st.rng_states = states.ctypes.data_as(C.POINTER(C.c_uint64))
            st._keep = states
        elif states_ptr is not None:
            st.rng_states = C.cast(C.c_void_p(states_ptr), C.POINTER(C.c_uint64))
        return st

    def render_device(self, cam, settings: abi.pt_settings, out_ptr: int, aux_ptr: int = 0, rays_ptr: int = 0,
                      stream: int = 0) -> None:
        """Enqueues a frame on `stream` with device buffers (no synchronisation)."""
        check(load().pt_render_device(self._h, C.byref(cam), C.byref(settings), C.c_void_p(out_ptr),
                                      C.c_void_p(aux_ptr or None), C.c_void_p(rays_ptr or None),
                                      C.c_void_p(stream or None)))

    def render_progressive(self, cam, settings: abi.pt_settings, progress=None):
        """pt_render_progressive: batches of growing spp summed in FP64.
        progress(done, total) -> truthy stops early. Returns (image, samples done, rays)."""
        out = np.empty((settings.height, settings.width, 3), np.float32)
        done, rays = C.c_int32(), C.c_uint64()
        cb = abi.PROGRESS_FN(lambda _u, d, t: int(bool(progress(d, t)))) if progress else abi.PROGRESS_FN()
        check(load().pt_render_progressive(self._h, C.byref(cam), C.byref(settings), _ptr(out), cb, None,
                                           C.byref(done), C.byref(rays)))
        return out, done.value, rays.value

    def sync(self, stream: int = 0) -> None:
        check(load().pt_sync(self._h, C.c_void_p(stream or None)))

    # -- ray queries --
    def trace_closest(self, rays: np.ndarray, tmin: float = 0.001, tmax: float = 1000.0) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.empty(rays.shape[0], abi.HIT_DTYPE)
        check(load().pt_trace_closest(self._h, _ptr(rays), rays.shape[0], tmin, tmax, _ptr(out)))
        return out

    def trace_any(self, rays: np.ndarray, tmin: float = 0.001, tmax: float = 1000.0) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.empty(rays.shape[0], np.uint8)
        check(load().pt_trace_any(self._h, _ptr(rays), rays.shape[0], tmin, tmax, _ptr(out)))
        return out

    def trace_count(self, rays: np.ndarray, tmin: float = 0.001, tmax: float = 1000.0) -> np.ndarray:
        """Per-kind traversal work summed over the rays: nodes, order entries, triangles, spheres, instances."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = (C.c_uint64 * 5)()
        check(load().pt_trace_count(self._h, _ptr(rays), rays.shape[0], tmin, tmax, out))
        return np.array(list(out), np.uint64)

    def trace_closest_device(self, rays_ptr: int, n: int, hits_ptr: int, tmin=0.001, tmax=1000.0, stream=0):
        check(load().pt_trace_closest_device(self._h, C.c_void_p(rays_ptr), n, tmin, tmax, C.c_void_p(hits_ptr),
                                             C.c_void_p(stream or None)))


# ---- the reference's row call -------------------------------------------------------
def render_row_linear(scene: Scene, cam, j: int, width: int, height: int, samples_per_pixel: int,
                      max_bounces: int, out: np.ndarray, seed: int, first_sample: int = 0,
                      aux: Optional[np.ndarray] = None) -> None:
    """render_row_linear (include/renderer.hpp:411-416): scanline j (from the
    bottom) into out (3 * width float32), aux (7 * width float32) if given."""
    if out.dtype != np.float32 or out.size < 3 * width or not out.flags.c_contiguous:
        raise ValueError("out must be a contiguous float32 array of 3 * width")
    if aux is not None and (aux.dtype != np.float32 or aux.size < 7 * width or not aux.flags.c_contiguous):
        raise ValueError("aux must be a contiguous float32 array of 7 * width")
    check(load().pt_render_row(scene.handle, C.byref(cam), j, width, height, samples_per_pixel, max_bounces,
                               _ptr(out), seed, first_sample, _ptr(aux)))


# ---- images ----------------------------------------------------------------------
def write_image(path: str, image: np.ndarray) -> None:
    """write_image (include/image_write.hpp:15-33): PFM for *.pfm, else PPM.
    image: H x W x 3 linear float32, top row first."""
    img = np.ascontiguousarray(image, np.float32)
    check(load().pt_write_image(path.encode(), img.shape[1], img.shape[0], _ptr(img)))


# ---- denoising ----------------------------------------------------------------------
def denoise_atrous(color: np.ndarray, albedo: np.ndarray, normal: np.ndarray, variance: np.ndarray) -> np.ndarray:
    """denoise (include/denoise.hpp:55-139) on the GPU; arrays H x W x {3,3,3,1}."""
    h, w = color.shape[:2]
    c = [np.ascontiguousarray(a, np.float32) for a in (color, albedo, normal, variance)]
    out = np.empty((h, w, 3), np.float32)
    check(load().pt_denoise_atrous(w, h, *[_ptr(a) for a in c], _ptr(out)))
    return out


# ---- batched rendering ------------------------------------------------------------
class Batch:
    """Many scenes rendered together (pt_batch_*): one device arena and, with
    PT_BATCH_ONE_LAUNCH, one persistent launch replayed from a CUDA graph.
    items: [(scene_with_desc, camera, width, height, spp, seed), ...] where the
    scene is a Generated (or anything with .desc_ptr)."""

    def __init__(self, items, strategy: int = abi.PT_BATCH_AUTO, max_bounces: int = 10):
        lib = load()
        self._keep = [it[0] for it in items]
        arr = (abi.pt_batch_item * len(items))()
        self.sizes = []
        for i, (scene, cam, w, h, spp, seed) in enumerate(items):
            arr[i].desc = scene.desc_ptr
            arr[i].camera = cam
            arr[i].width, arr[i].height, arr[i].spp, arr[i].max_bounces, arr[i].seed = w, h, spp, max_bounces, seed
            self.sizes.append((w, h, spp))
        h = C.c_void_p()
        check(lib.pt_batch_create(arr, len(items), strategy, C.byref(h)))
        self._h = h

    def render(self, stream: int = 0, count_rays: bool = True):
        rays = C.c_uint64()
        check(load().pt_batch_render(self._h, C.c_void_p(stream or None), C.byref(rays) if count_rays else None))
        return rays.value

    def image(self, i: int) -> np.ndarray:
        w, h, _ = self.sizes[i]
        out = np.empty((h, w, 3), np.float32)
        check(load().pt_batch_download(self._h, i, _ptr(out)))
        return out

    def scene_times(self) -> np.ndarray:
        ms = (C.c_double * len(self.sizes))()
        check(load().pt_batch_scene_times(self._h, ms))
        return np.array(list(ms))

    def info(self) -> abi.pt_batch_info:
        i = abi.pt_batch_info()
        check(load().pt_batch_get_info(self._h, C.byref(i)))
        return i

    def close(self):
        if getattr(self, "_h", None):
            load().pt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_scenes(n: int = 64, first_seed: int = 1):
    """The batched workload: n scenes from seeds first_seed.. of the batch
    generator (random spheres with 10..2000 spheres or the room with a
    2..7-subdivision icosphere; 256..1024 square; 4/16/64 spp)."""
    out = []
    for s in range(first_seed, first_seed + n):
        g = Generated(abi.PT_GEN_BATCH_SCENE, seed=s)
        out.append((g, g.camera, g.width, g.height, g.spp, s))
    return out
