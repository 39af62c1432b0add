"""ctypes mirror of include/photon_cuda.h: structs, numpy dtypes of the array
element types, and the loader of libphoton_cuda.so.

The library is built in-tree (python -m photon_tracer_b200.build). Loading
fails loudly when it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphoton_cuda.so")

# status codes
PT_OK = 0
PT_ERR_INVALID_ARG = 1
PT_ERR_OUT_OF_MEMORY = 2
PT_ERR_STACK_OVERFLOW = 3
PT_ERR_QUEUE_OVERFLOW = 4
PT_ERR_TIMEOUT = 5
PT_ERR_CUDA = 6
PT_ERR_NO_DEVICE = 7
PT_ERR_UNSUPPORTED = 8
STATUS_NAMES = {0: "PT_OK", 1: "PT_ERR_INVALID_ARG", 2: "PT_ERR_OUT_OF_MEMORY", 3: "PT_ERR_STACK_OVERFLOW",
                4: "PT_ERR_QUEUE_OVERFLOW", 5: "PT_ERR_TIMEOUT", 6: "PT_ERR_CUDA", 7: "PT_ERR_NO_DEVICE",
                8: "PT_ERR_UNSUPPORTED"}

PT_MAT_LAMBERTIAN, PT_MAT_METAL, PT_MAT_DIELECTRIC, PT_MAT_DIFFUSE_LIGHT = 0, 1, 2, 3
PT_NO_MATERIAL = 0xFFFFFFFF
PT_MODE_AUTO, PT_MODE_MEGAKERNEL, PT_MODE_WAVEFRONT = 0, 1, 2
PT_RNG_SAMPLE, PT_RNG_SNAPSHOT = 0, 1
PT_FLAG_NEE_EXTENDED = 1
PT_HIT_NONE, PT_HIT_LARGE, PT_HIT_SPHERE, PT_HIT_TRIANGLE, PT_HIT_INSTANCE = 0, 1, 2, 3, 4

PT_GEN_REF_MATERIALS = 0
PT_GEN_REF_FIELD = 1
PT_GEN_REF_ROOM = 3
PT_GEN_RANDOM_SPHERES = 10
PT_GEN_ROOM_MESH = 11
PT_GEN_INSTANCES = 12
PT_GEN_BATCH_SCENE = 13
PT_GEN_TEXTURED = 14
PT_GEN_MESH_LIGHT = 15

PT_ATROUS_NOALLOC_MAX_PIXELS = 262144  # the built-in scratch of pt_denoise_atrous_device_noalloc

F3 = C.c_float * 3


class pt_material(C.Structure):
    _fields_ = [("type", C.c_uint32), ("albedo", F3), ("emission", F3), ("fuzz", C.c_float), ("ior", C.c_float),
                ("texture", C.c_uint32)]


class pt_texture(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("rgb", C.POINTER(C.c_uint8))]


class pt_sphere(C.Structure):
    _fields_ = [("center", F3), ("radius", C.c_float), ("material", C.c_uint32)]


class pt_triangle(C.Structure):
    _fields_ = [("p0", F3), ("e1", F3), ("e2", F3), ("n0", F3), ("n1", F3), ("n2", F3), ("face_normal", F3),
                ("p1", F3), ("p2", F3), ("material", C.c_uint32), ("uv", C.c_float * 6)]


class pt_affine(C.Structure):
    _fields_ = [("m", (C.c_float * 3) * 3), ("t", F3)]


class pt_bvh_node(C.Structure):
    _fields_ = [("lo", (C.c_float * 4) * 3), ("hi", (C.c_float * 4) * 3), ("first", C.c_uint32 * 4),
                ("count", C.c_uint32 * 4)]


class pt_bvh(C.Structure):
    _fields_ = [("nodes", C.POINTER(pt_bvh_node)), ("n_nodes", C.c_uint32), ("order", C.POINTER(C.c_uint32)),
                ("n_order", C.c_uint32)]


class pt_mesh(C.Structure):
    _fields_ = [("triangles", C.POINTER(pt_triangle)), ("n_triangles", C.c_uint32), ("tree", pt_bvh)]


class pt_instance(C.Structure):
    _fields_ = [("mesh", C.c_uint32), ("material", C.c_uint32), ("to_world", pt_affine), ("to_object", pt_affine)]


class pt_scene_desc(C.Structure):
    _fields_ = [("materials", C.POINTER(pt_material)), ("n_materials", C.c_uint32),
                ("spheres", C.POINTER(pt_sphere)), ("n_spheres", C.c_uint32),
                ("large_spheres", C.POINTER(pt_sphere)), ("n_large_spheres", C.c_uint32),
                ("triangles", C.POINTER(pt_triangle)), ("n_triangles", C.c_uint32),
                ("meshes", C.POINTER(pt_mesh)), ("n_meshes", C.c_uint32),
                ("instances", C.POINTER(pt_instance)), ("n_instances", C.c_uint32),
                ("flat_tree", pt_bvh), ("instance_tree", pt_bvh),
                ("lights", C.POINTER(C.c_uint32)), ("n_lights", C.c_uint32),
                ("sky", C.c_int32), ("sample_lights", C.c_int32), ("use_bvh", C.c_int32),
                ("textures", C.POINTER(pt_texture)), ("n_textures", C.c_uint32)]


class pt_scene_info(C.Structure):
    _fields_ = [("n_nodes", C.c_uint32), ("n_slots", C.c_uint32), ("max_depth", C.c_uint32),
                ("stack_entries", C.c_uint32), ("device_bytes", C.c_uint64)]


class pt_camera(C.Structure):
    _fields_ = [("origin", F3), ("lower_left", F3), ("horizontal", F3), ("vertical", F3)]


class pt_settings(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_bounces", C.c_int32),
                ("seed", C.c_uint64), ("first_sample", C.c_int32), ("mode", C.c_int32), ("rng", C.c_int32),
                ("flags", C.c_int32), ("rng_states", C.POINTER(C.c_uint64))]


class pt_hit(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("index", C.c_uint32), ("sub", C.c_uint32), ("t", C.c_float),
                ("u", C.c_float), ("v", C.c_float)]


class pt_gen_params(C.Structure):
    _fields_ = [("kind", C.c_int32), ("param", C.c_int32), ("seed", C.c_uint64), ("use_bvh", C.c_int32),
                ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32)]


class pt_batch_item(C.Structure):
    _fields_ = [("desc", C.POINTER(pt_scene_desc)), ("camera", pt_camera), ("width", C.c_int32), ("height", C.c_int32),
                ("spp", C.c_int32), ("max_bounces", C.c_int32), ("seed", C.c_uint64)]


class pt_batch_info(C.Structure):
    _fields_ = [("n_scenes", C.c_uint32), ("strategy", C.c_int32), ("threads", C.c_int32), ("tuned", C.c_int32),
                ("total_pixels", C.c_uint64), ("total_samples", C.c_uint64), ("device_bytes", C.c_uint64),
                ("tune_ms", C.c_double * 8)]


PT_BATCH_AUTO, PT_BATCH_ONE_LAUNCH, PT_BATCH_PER_SCENE_MEGA, PT_BATCH_PER_SCENE_WAVE = 0, 1, 2, 3

HIT_DTYPE = np.dtype([("kind", "<u4"), ("index", "<u4"), ("sub", "<u4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
NODE_DTYPE = np.dtype([("lo", "<f4", (3, 4)), ("hi", "<f4", (3, 4)), ("first", "<u4", (4,)), ("count", "<u4", (4,))])
assert HIT_DTYPE.itemsize == C.sizeof(pt_hit)
assert NODE_DTYPE.itemsize == C.sizeof(pt_bvh_node) == 128

P = C.c_void_p
ST = C.c_int32
SIZE = C.c_size_t

# (name, restype, argtypes) of every entry point include/photon_cuda.h declares.
PROGRESS_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_int32)

PROTOTYPES = [
    ("pt_last_error", C.c_char_p, []),
    ("pt_version", C.c_char_p, []),
    ("pt_scene_create", ST, [C.POINTER(pt_scene_desc), C.POINTER(P)]),
    ("pt_scene_destroy", ST, [P]),
    ("pt_scene_get_info", ST, [P, C.POINTER(pt_scene_info)]),
    ("pt_camera_look_at", ST, [F3, F3, C.c_double, C.c_double, C.POINTER(pt_camera)]),
    ("pt_render", ST, [P, C.POINTER(pt_camera), C.POINTER(pt_settings), P, P, C.POINTER(C.c_uint64)]),
    ("pt_render_device", ST, [P, C.POINTER(pt_camera), C.POINTER(pt_settings), P, P, P, P]),
    ("pt_render_row", ST, [P, C.POINTER(pt_camera), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_uint64,
                           C.c_int, P]),
    ("pt_sync", ST, [P, P]),
    ("pt_trace_closest", ST, [P, P, SIZE, C.c_float, C.c_float, P]),
    ("pt_trace_any", ST, [P, P, SIZE, C.c_float, C.c_float, P]),
    ("pt_trace_closest_device", ST, [P, P, SIZE, C.c_float, C.c_float, P, P]),
    ("pt_trace_any_device", ST, [P, P, SIZE, C.c_float, C.c_float, P, P]),
    ("pt_render_progressive", ST, [P, C.POINTER(pt_camera), C.POINTER(pt_settings), P, PROGRESS_FN, P,
                                   C.POINTER(C.c_int32), C.POINTER(C.c_uint64)]),
    ("pt_primary_depth_device", ST, [P, C.POINTER(pt_camera), C.c_int, C.c_int, P, P]),
    ("pt_trace_count", ST, [P, P, SIZE, C.c_float, C.c_float, C.POINTER(C.c_uint64)]),
    ("pt_affine_inverse", ST, [C.POINTER(pt_affine), C.POINTER(pt_affine)]),
    ("pt_triangle_init", ST, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                              C.c_uint32, C.POINTER(pt_triangle)]),
    ("pt_bvh_build", ST, [P, C.c_uint32, C.POINTER(C.POINTER(pt_bvh_node)), C.POINTER(C.c_uint32),
                          C.POINTER(C.POINTER(C.c_uint32))]),
    ("pt_bvh_build_gpu", ST, [P, C.c_uint32, C.POINTER(C.POINTER(pt_bvh_node)), C.POINTER(C.c_uint32),
                              C.POINTER(C.POINTER(C.c_uint32))]),
    ("pt_free", None, [P]),
    ("pt_denoise_atrous", ST, [C.c_int, C.c_int, P, P, P, P, P]),
    ("pt_denoise_atrous_device", ST, [C.c_int, C.c_int, P, P, P, P, P, P, P]),
    ("pt_denoise_atrous_scratch_floats", SIZE, [C.c_int, C.c_int]),
    ("pt_denoise_atrous_device_noalloc", ST, [C.c_int, C.c_int, P, P, P, P, P, P]),
    ("pt_measure_l2_read", ST, [C.c_size_t, C.c_int, C.POINTER(C.c_double)]),
    ("pt_unet_create", ST, [C.c_uint64, C.POINTER(P)]),
    ("pt_unet_destroy", ST, [P]),
    ("pt_unet_num_params", SIZE, [P]),
    ("pt_unet_get_params", ST, [P, P]),
    ("pt_unet_set_params", ST, [P, P]),
    ("pt_unet_set_tensor_cores", ST, [P, C.c_int]),
    ("pt_unet_sync", ST, [P, P]),
    ("pt_unet_forward", ST, [P, C.c_int, C.c_int, C.c_int, P, P, P]),
    ("pt_unet_train_step", ST, [P, C.c_int, C.c_int, C.c_int, P, P, C.c_float, C.POINTER(C.c_float), P]),
    ("pt_unet_loss_grads", ST, [P, C.c_int, C.c_int, C.c_int, P, P, C.POINTER(C.c_float), P, P]),
    ("pt_denoise_unet", ST, [P, C.c_int, C.c_int, P, P, P, P, P]),
    ("pt_accumulate_pass", ST, [P, SIZE, C.c_double, P, P]),
    ("pt_write_image", ST, [C.c_char_p, C.c_int, C.c_int, P]),
    ("pt_to_display", C.c_uint8, [C.c_float]),
    ("pt_batch_create", ST, [C.POINTER(pt_batch_item), C.c_uint32, C.c_int32, C.POINTER(P)]),
    ("pt_batch_render", ST, [P, P, C.POINTER(C.c_uint64)]),
    ("pt_batch_output", ST, [P, C.c_uint32, C.POINTER(P)]),
    ("pt_batch_download", ST, [P, C.c_uint32, P]),
    ("pt_batch_scene_times", ST, [P, C.POINTER(C.c_double)]),
    ("pt_batch_get_info", ST, [P, C.POINTER(pt_batch_info)]),
    ("pt_batch_destroy", ST, [P]),
    ("pt_generate", ST, [C.POINTER(pt_gen_params), C.POINTER(P)]),
    ("pt_generated_desc", C.POINTER(pt_scene_desc), [P]),
    ("pt_generated_camera", C.POINTER(pt_camera), [P]),
    ("pt_generated_free", None, [P]),
    ("pt_generate_rays", ST, [C.c_uint64, F3, F3, SIZE, P]),
]

_lib = None


def load() -> C.CDLL:
    """The loaded libphoton_cuda.so with prototypes set. Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m photon_tracer_b200.build` "
                           "(the CUDA library is required; there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in PROTOTYPES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class PhotonError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(status: int) -> None:
    if status != PT_OK:
        msg = load().pt_last_error()
        raise PhotonError(status, msg.decode() if msg else "")


def f3(v) -> "C.Array":
    return F3(*[float(x) for x in v])

TRIANGLE_DTYPE = np.dtype([("p0", "<f4", 3), ("e1", "<f4", 3), ("e2", "<f4", 3), ("n0", "<f4", 3), ("n1", "<f4", 3),
                           ("n2", "<f4", 3), ("face_normal", "<f4", 3), ("p1", "<f4", 3), ("p2", "<f4", 3),
                           ("material", "<u4"), ("uv", "<f4", 6)])
SPHERE_DTYPE = np.dtype([("center", "<f4", 3), ("radius", "<f4"), ("material", "<u4")])
AFFINE_DTYPE = np.dtype([("m", "<f4", (3, 3)), ("t", "<f4", 3)])
INSTANCE_DTYPE = np.dtype([("mesh", "<u4"), ("material", "<u4"), ("to_world", AFFINE_DTYPE),
                           ("to_object", AFFINE_DTYPE)])
MATERIAL_DTYPE = np.dtype([("type", "<u4"), ("albedo", "<f4", 3), ("emission", "<f4", 3), ("fuzz", "<f4"),
                           ("ior", "<f4"), ("texture", "<u4")])
assert TRIANGLE_DTYPE.itemsize == C.sizeof(pt_triangle)
assert SPHERE_DTYPE.itemsize == C.sizeof(pt_sphere)
assert INSTANCE_DTYPE.itemsize == C.sizeof(pt_instance)
assert MATERIAL_DTYPE.itemsize == C.sizeof(pt_material)


def view(ptr, n: int, dtype: np.dtype) -> np.ndarray:
    """A numpy view of n elements of dtype at a ctypes pointer (empty when n == 0)."""
    if n == 0 or not ptr:
        return np.zeros(0, dtype)
    raw = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), (n * dtype.itemsize,))
    return raw.view(dtype)


def desc_arrays(desc: pt_scene_desc) -> dict:
    """numpy views of a scene description's arrays (no copies)."""
    return {
        "materials": view(desc.materials, desc.n_materials, MATERIAL_DTYPE),
        "spheres": view(desc.spheres, desc.n_spheres, SPHERE_DTYPE),
        "large_spheres": view(desc.large_spheres, desc.n_large_spheres, SPHERE_DTYPE),
        "triangles": view(desc.triangles, desc.n_triangles, TRIANGLE_DTYPE),
        "meshes": [view(desc.meshes[m].triangles, desc.meshes[m].n_triangles, TRIANGLE_DTYPE)
                   for m in range(desc.n_meshes)],
        "instances": view(desc.instances, desc.n_instances, INSTANCE_DTYPE),
    }
