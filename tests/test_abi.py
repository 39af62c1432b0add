"""The C ABI: the library loads, exports every entry point include/photon_cuda.h
declares, its structs have the sizes the header gives them, and calls fail
with status codes (never exceptions or crashes) on bad input. CPU only."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "photon_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pt_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("pt_scene_create", "pt_render", "pt_render_row", "pt_trace_closest", "pt_trace_any",
                 "pt_denoise_atrous", "pt_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(built):
    lib = C.CDLL(os.path.join(ROOT, "photon_tracer_b200", "libphoton_cuda.so"))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_prototypes_cover_header(built):
    from photon_tracer_b200 import abi
    assert sorted(n for n, _, _ in abi.PROTOTYPES) == declared_functions()


def test_struct_sizes_match_c(built, tmp_path):
    """ctypes mirrors against sizeof/offsetof from a C compile of the header."""
    from photon_tracer_b200 import abi
    structs = ["pt_material", "pt_sphere", "pt_triangle", "pt_affine", "pt_bvh_node", "pt_bvh", "pt_mesh",
               "pt_instance", "pt_scene_desc", "pt_scene_info", "pt_camera", "pt_settings", "pt_hit", "pt_gen_params",
               "pt_batch_item", "pt_batch_info", "pt_texture"]
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "photon_cuda.h"\nint main(void){\n' +
                   "".join(f'printf("{s} %zu\\n", sizeof({s}));\n' for s in structs) +
                   'printf("off_settings_states %zu\\n", offsetof(pt_settings, rng_states));\n'
                   'printf("off_desc_use_bvh %zu\\n", offsetof(pt_scene_desc, use_bvh));\n'
                   'printf("off_desc_textures %zu\\n", offsetof(pt_scene_desc, textures));\n'
                   'printf("off_tri_uv %zu\\n", offsetof(pt_triangle, uv));\nreturn 0;}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for s in structs:
        assert int(out[s]) == C.sizeof(getattr(abi, s)), s
    assert int(out["off_settings_states"]) == abi.pt_settings.rng_states.offset
    assert int(out["off_desc_use_bvh"]) == abi.pt_scene_desc.use_bvh.offset
    assert int(out["off_desc_textures"]) == abi.pt_scene_desc.textures.offset
    assert int(out["off_tri_uv"]) == abi.pt_triangle.uv.offset


def test_version_and_error_text(built):
    lib = built.load()
    assert b"sm_100a" in lib.pt_version()
    assert lib.pt_last_error() is not None


def test_invalid_arguments_return_codes(built):
    from photon_tracer_b200 import abi
    lib = built.load()
    assert lib.pt_scene_create(None, None) == abi.PT_ERR_INVALID_ARG
    assert b"null" in lib.pt_last_error()
    assert lib.pt_render(None, None, None, None, None, None) == abi.PT_ERR_INVALID_ARG
    assert lib.pt_trace_closest(None, None, 0, 0.0, 1.0, None) == abi.PT_ERR_INVALID_ARG
    assert lib.pt_denoise_atrous(0, 0, None, None, None, None, None) == abi.PT_ERR_INVALID_ARG
    assert lib.pt_scene_destroy(None) == abi.PT_OK
    params = abi.pt_gen_params(kind=999)
    h = C.c_void_p()
    assert lib.pt_generate(C.byref(params), C.byref(h)) == abi.PT_ERR_INVALID_ARG


def test_scene_validation_before_device(built):
    """Invalid descriptions are refused by the host-side repack, before any
    device is touched, with PT_ERR_INVALID_ARG and a message naming the
    field (so the same answer comes with or without a GPU)."""
    from photon_tracer_b200 import abi
    lib = built.load()
    mat = abi.pt_material(type=0, albedo=abi.F3(0.5, 0.5, 0.5))
    px = (C.c_uint8 * 3)(1, 2, 3)

    def create(**kw):
        keep = []

        def arr(t, items):
            a = (t * max(1, len(items)))(*items)
            keep.append(a)
            return a
        mats = kw.pop("materials", [mat])
        sph = kw.pop("spheres", [])
        tris = kw.pop("triangles", [])
        meshes = kw.pop("meshes", [])
        inst = kw.pop("instances", [])
        tex = kw.pop("textures", [])
        lights = kw.pop("lights", None)
        d = abi.pt_scene_desc(materials=arr(abi.pt_material, mats), n_materials=len(mats),
                              spheres=arr(abi.pt_sphere, sph), n_spheres=len(sph),
                              triangles=arr(abi.pt_triangle, tris), n_triangles=len(tris),
                              meshes=arr(abi.pt_mesh, meshes), n_meshes=len(meshes),
                              instances=arr(abi.pt_instance, inst), n_instances=len(inst),
                              textures=arr(abi.pt_texture, tex), n_textures=len(tex), use_bvh=1, sky=1)
        if lights is not None:
            d.lights = arr(C.c_uint32, lights)
            d.n_lights = len(lights)
        h = C.c_void_p()
        st = lib.pt_scene_create(C.byref(d), C.byref(h))
        return st, lib.pt_last_error().decode()

    tri = built.triangle((0, 0, 0), (1, 0, 0), (0, 1, 0), material=3)
    mesh_tri = (abi.pt_triangle * 1)(built.triangle((0, 0, 0), (1, 0, 0), (0, 1, 0)))
    mesh = abi.pt_mesh(triangles=mesh_tri, n_triangles=1)
    cases = [
        (dict(spheres=[abi.pt_sphere(radius=1.0, material=7)]), "sphere: material"),
        (dict(triangles=[tri]), "triangle: material"),
        (dict(materials=[abi.pt_material(type=9)]), "unknown type"),
        (dict(materials=[abi.pt_material(type=0, texture=2)], textures=[abi.pt_texture(1, 1, px)]), "texture out"),
        (dict(textures=[abi.pt_texture(0, 4, px)]), "texture: empty"),
        (dict(meshes=[mesh], instances=[abi.pt_instance(mesh=3)]), "instance: mesh"),
        (dict(meshes=[mesh], instances=[abi.pt_instance(mesh=0, material=5)]), "instance: material"),
        (dict(spheres=[abi.pt_sphere(radius=1.0)], lights=[4]), "light: sphere"),
    ]
    for kw, words in cases:
        st, msg = create(**kw)
        assert st == abi.PT_ERR_INVALID_ARG and words in msg, (words, st, msg)


def test_no_device_is_an_error_not_a_fallback(built):
    """Without a GPU the library refuses to create scenes (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from photon_tracer_b200 import abi
    g = built.Generated(abi.PT_GEN_REF_ROOM)
    with pytest.raises(built.PhotonError) as e:
        built.Scene(g)
    assert e.value.status == abi.PT_ERR_NO_DEVICE


def test_camera_matches_reference(built):
    """pt_camera_look_at with 16:9 is the reference's camera bit for bit."""
    from oracle.oracle import ref_available, ref_camera
    if not ref_available():
        pytest.skip("reference harness absent")
    for frm, at, vfov in [((0, 0, 0), (0, 0, -1), 90.0), ((13, 2, 3), (0, 0, 0), 20.0),
                          ((0, 0, 0.3), (0, -0.15, -3.0), 62.0), ((0, 1.0, 1.2), (0, -0.3, -1.2), 55.0)]:
        mine = built.camera_look_at(frm, at, vfov)
        ref = ref_camera(frm, at, vfov)
        assert bytes(mine) == bytes(ref)


def test_rays_generator_is_deterministic(built):
    a = built.generate_rays(1, [-1, -1, -1], [1, 1, 1], 1000)
    b = built.generate_rays(1, [-1, -1, -1], [1, 1, 1], 1000)
    assert np.array_equal(a, b)
    assert np.all(np.abs(a[:, :3]) <= 1)
    n = np.linalg.norm(a[:, 3:].astype(np.float64), axis=1)
    assert np.allclose(n, 1, atol=1e-6)


def test_geometry_bridge_compiles_and_reports_no_device(built):
    """include/photon_cuda_geometry.hpp compiled against the reference's own
    headers (oracle/_ref/shim_check): without a GPU the upload answers
    PT_ERR_NO_DEVICE instead of falling back to anything."""
    import json
    import torch
    shim = os.path.join(ROOT, "oracle", "_ref", "shim_check")
    if not os.path.exists(shim):
        pytest.skip("reference checkout absent: the bridge check is not built")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present (the GPU test runs the bridge)")
    res = subprocess.run([shim, "3"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 3
    assert json.loads(res.stdout)["upload"] == 7


def test_write_image_matches_reference(built, tmp_path):
    """PFM and PPM bytes identical to the reference's write_image."""
    from oracle.oracle import ref_available, ref_lib
    rng = np.random.default_rng(4)
    img = rng.uniform(-0.2, 1.6, (27, 48, 3)).astype(np.float32)
    img[0, :4] = [[0, 0, 0], [1, 1, 1], [0.998, 0.999, 1.0], [4.0, 1e-9, 0.25]]
    for ext in ("pfm", "ppm"):
        mine = tmp_path / f"mine.{ext}"
        built.write_image(str(mine), img)
        data = mine.read_bytes()
        if ext == "pfm":
            head = b"PF\n48 27\n-1.0\n"
            assert data.startswith(head)
            back = np.frombuffer(data[len(head):], np.float32).reshape(27, 48, 3)[::-1]
            assert np.array_equal(back, img)
        if ref_available():
            theirs = tmp_path / f"ref.{ext}"
            assert ref_lib().ref_write_image(str(theirs).encode(), 48, 27, img.ctypes.data_as(C.c_void_p)) == 1
            assert data == theirs.read_bytes()
