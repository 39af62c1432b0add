"""photon_tracer_b200: the render hot path of photon_tracer on one B200.

libphoton_cuda.so (built in-tree by ``python -m photon_tracer_b200.build``)
holds the CUDA kernels and the C ABI (include/photon_cuda.h); this package is
the Python host side over it. There is no CPU fallback: without the library,
or without an sm_100 GPU, calls raise.
"""
from . import abi
from .abi import PhotonError, load
from .api import (Batch, Generated, Scene, SceneInfo, affine_inverse, batch_scenes, bvh_build, camera_look_at,
                  denoise_atrous, generate_rays, render_row_linear, triangle, write_image)

__all__ = ["abi", "load", "PhotonError", "Batch", "affine_inverse", "batch_scenes", "Generated", "Scene", "SceneInfo",
           "bvh_build", "camera_look_at",
           "denoise_atrous", "generate_rays", "render_row_linear", "triangle", "write_image"]
