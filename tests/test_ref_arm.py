"""The benchmark's reference arm renders the room-mesh frame with the
reference's own code and no product code loaded (oracle/ref_arm.py): its
scene, built through the reference's classes, must be the product's
generated scene byte for byte, and its camera the product's camera."""
import ast
import os

import numpy as np
import pytest

from conftest import ROOT


def test_ref_arm_module_imports_no_product_code():
    tree = ast.parse(open(os.path.join(ROOT, "oracle", "ref_arm.py")).read())
    names = [a.name for n in ast.walk(tree) if isinstance(n, ast.Import) for a in n.names]
    names += [n.module or "" for n in ast.walk(tree) if isinstance(n, ast.ImportFrom)]
    assert not any(m.startswith(("photon_tracer_b200", "oracle.oracle")) for m in names), names


def test_reference_built_frame_equals_the_generated_one(built):
    from oracle import ref_arm
    from oracle.oracle import reference_trees, Reference
    from photon_tracer_b200 import abi
    if not ref_arm.available():
        pytest.skip("reference harness absent")
    import ctypes as C
    frame = ref_arm.RoomMeshFrame()
    L = frame.lib
    L.ref_world_desc.restype = C.POINTER(abi.pt_scene_desc)
    L.ref_world_desc.argtypes = [C.c_void_p]
    L.ref_world_camera.restype = C.POINTER(abi.pt_camera)
    L.ref_world_camera.argtypes = [C.c_void_p]
    mine = L.ref_world_desc(frame.h).contents
    g = built.Generated(abi.PT_GEN_ROOM_MESH, seed=ref_arm.SEED, param=ref_arm.SUBDIV)
    a, b = abi.desc_arrays(mine), abi.desc_arrays(g.desc)
    assert bytes(L.ref_world_camera(frame.h).contents) == bytes(g.camera)
    for k in ("spheres", "triangles"):
        x, y = a[k].copy(), b[k].copy()
        # materials are numbered in a different order: compare them by value
        assert a["materials"][x["material"]].tobytes() == b["materials"][y["material"]].tobytes(), k
        x["material"] = 0
        y["material"] = 0
        assert x.tobytes() == y.tobytes(), k
    assert (mine.sky, mine.sample_lights, mine.use_bvh) == (g.desc.sky, g.desc.sample_lights, g.desc.use_bvh)
    # and the reference builds the same trees from either description
    t1 = reference_trees(Reference(mine), mine).arrays[0]
    t2 = reference_trees(Reference(g.desc), g.desc).arrays[0]
    assert t1[0].tobytes() == t2[0].tobytes() and np.array_equal(t1[1], t2[1])
    frame.close()


def test_row_set_render_counts_rays(built):
    from oracle import ref_arm
    if not ref_arm.available():
        pytest.skip("reference harness absent")
    frame = ref_arm.RoomMeshFrame()
    frame.rows = frame.rows[:4]
    import ctypes as C
    frame._rows = (C.c_int * 4)(*frame.rows)
    rays, secs = frame.render_rows(2)
    assert rays > 4 * ref_arm.WIDTH * ref_arm.SPP and secs > 0
