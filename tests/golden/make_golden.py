"""Writes the golden fixtures under tests/golden/ from the reference itself.

Run in a checkout that has the reference (the directory oracle/build.py
names: PT_REFERENCE_DIR, else its default) with oracle/_ref built
(python oracle/build.py). The
fixtures let the tests pin the CPU restatement on machines without the
reference:

* reference_blocks.npz -- the reference's own statistical render fixture
  (tests/reference.json: per-20x20-block mean linear colour and sigma over 16
  seeds, 960x540 at 200 spp) for the scenes this path renders: materials,
  field, room, teapot, crowd (which the flattened crowd must also match) and
  spot crowd;
* ref_hits_*.npz      -- rays and the reference's closest/any hits on them;
* ref_render_*.npz    -- small renders by the reference's own per-row stream,
  with the xoshiro state captured before every sample's path;
* ref_trees.json      -- digests of the trees the reference's geometry::build
  makes for every scene generator;
* ref_denoise.npz     -- the reference's a-trous denoise of a small render of
  its own (colour, albedo, normal, per-pixel luminance variance) and of
  seeded random planes;
* ref_edge_hits.npz   -- the reference's closest/any hits for rays with
  infinite, signed-zero, denormal and huge components (room scene), and on
  the hand-made scenes with NaN and huge coordinates (tests/handmade.py);
* ref_material_renders.npz -- the reference's renders (24x16, 4 spp, image,
  guides, ray count, and the xoshiro state before every sample's path) of
  four random-material scenes (tests/handmade.py: metal fuzz above 1, ior at
  and below 1, negative radii, emitters);
* ref_scene_{teapot,crowd,spot_crowd}.npz -- the reference's OBJ scenes as its
  CLI builds them (--mesh; --crowd 8; --crowd 6 --obj models/spot/spot.obj
  --turn 150) from the models in its checkout, in the compact form of
  tests/scene_fixture.py, with digests of the trees geometry::build made; and
  their statistical fixtures added to reference_blocks.npz;
* ref_converge_{random_spheres,room_mesh,instances}.npz -- the reference's own
  renders of the 400x225 16-spp random-spheres frame, the 1024x1024 64-spp
  room-mesh frame and the 1920x1080 32-spp 10,000-instance frame over 16
  seeds: per-seed image means and per-20x20-block means and sigmas, for the
  0.1% convergence check.

    python tests/golden/make_golden.py [--only NAME ...]

NAME is one of blocks, hits, renders, trees, denoise, edge, materials,
obj_scenes, converge (default: all).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import photon_tracer_b200 as pt  # noqa: E402
from photon_tracer_b200 import abi  # noqa: E402
from oracle.build import REFERENCE  # noqa: E402
from oracle.oracle import Reference, reference_trees  # noqa: E402

if not os.path.isdir(os.path.join(REFERENCE, "include")):
    sys.exit(f"make_golden.py needs the reference checkout: set PT_REFERENCE_DIR (tried {REFERENCE})")

# (name, generator kind, param, ray box) of the hit fixtures
HIT_CASES = [
    ("room_mesh", abi.PT_GEN_ROOM_MESH, 6, ([-1, -1, -1], [1, 1, 1]), 8192),
    ("random_spheres", abi.PT_GEN_RANDOM_SPHERES, 0, ([-12, 0, -12], [12, 3, 12]), 8192),
    ("ref_room", abi.PT_GEN_REF_ROOM, 0, ([-1.75, -1, -3.5], [1.75, 1, 0.5]), 4096),
    ("instances", abi.PT_GEN_INSTANCES, 400, ([-30, 0, -30], [30, 6, 30]), 4096),
]
RENDER_CASES = [
    ("room_mesh", abi.PT_GEN_ROOM_MESH, 6, 32, 32, 2),
    ("random_spheres", abi.PT_GEN_RANDOM_SPHERES, 0, 40, 23, 2),
    ("ref_field", abi.PT_GEN_REF_FIELD, 0, 40, 23, 2),
    ("instances", abi.PT_GEN_INSTANCES, 400, 32, 18, 1),
    ("textured", abi.PT_GEN_TEXTURED, 0, 48, 27, 2),
]
TREE_CASES = [("ref_materials", abi.PT_GEN_REF_MATERIALS, 0), ("ref_field", abi.PT_GEN_REF_FIELD, 0),
              ("ref_room", abi.PT_GEN_REF_ROOM, 0), ("random_spheres", abi.PT_GEN_RANDOM_SPHERES, 0),
              ("room_mesh", abi.PT_GEN_ROOM_MESH, 6), ("instances", abi.PT_GEN_INSTANCES, 0)]


def tree_digest(trees) -> list:
    out = []
    for t in trees.arrays:
        if t is None:
            out.append(None)
        else:
            h = hashlib.sha256(t[0].tobytes() + t[1].tobytes()).hexdigest()
            out.append([int(len(t[0])), int(len(t[1])), h])
    return out


def write_denoise():
    from oracle.oracle import ref_denoise
    g = pt.Generated(abi.PT_GEN_ROOM_MESH, seed=1, param=3)
    r = Reference(g.desc)
    img, aux, _ = r.render(g.camera, 48, 32, 4, 10, seed=5, aux=True)
    lum = 0.2126 * img[..., 0] + 0.7152 * img[..., 1] + 0.0722 * img[..., 2]
    cases = {"render": (img, aux[..., 0:3], aux[..., 3:6], np.maximum(aux[..., 6] - lum * lum, 0))}
    rng = np.random.default_rng(7)
    cases["random"] = (rng.random((32, 45, 3), dtype=np.float32) * 3, rng.random((32, 45, 3), dtype=np.float32),
                       rng.normal(size=(32, 45, 3)).astype(np.float32), rng.random((32, 45), dtype=np.float32))
    arrays = {}
    for name, (c, al, nrm, var) in cases.items():
        c, al, nrm, var = (np.ascontiguousarray(x, np.float32) for x in (c, al, nrm, var))
        arrays.update({f"{name}_color": c, f"{name}_albedo": al, f"{name}_normal": nrm, f"{name}_variance": var,
                       f"{name}_out": ref_denoise(c, al, nrm, var)})
    np.savez_compressed(os.path.join(HERE, "ref_denoise.npz"), **arrays)


def write_edge_hits():
    sys.path.insert(0, os.path.dirname(HERE))
    from handmade import adversarial_rays, non_finite_scene, non_finite_spheres
    arrays = {}
    g = pt.Generated(abi.PT_GEN_ROOM_MESH, seed=2, param=3)
    r = Reference(g.desc)
    rays = adversarial_rays(9, 20000)[:5000]
    hits, _ = r.trace_closest(rays)
    arrays.update(adversarial_rays=rays, adversarial_hits=hits.view(np.uint32).reshape(-1, 6),
                  adversarial_occluded=r.trace_any(rays))
    for name, make in (("nan_triangles", non_finite_scene), ("nan_spheres", non_finite_spheres)):
        d, rays = make(pt)
        rays = rays[:5000]
        r = Reference(d.desc)
        hits, _ = r.trace_closest(rays)
        arrays.update({f"{name}_rays": rays, f"{name}_hits": hits.view(np.uint32).reshape(-1, 6),
                       f"{name}_occluded": r.trace_any(rays)})
    np.savez_compressed(os.path.join(HERE, "ref_edge_hits.npz"), **arrays)


def write_material_renders():
    sys.path.insert(0, os.path.dirname(HERE))
    from handmade import random_material_scene
    arrays = {}
    for seed in range(4):
        d, cam = random_material_scene(pt, 500 + seed)
        r = Reference(d.desc)
        img, aux, rays = r.render(cam, 24, 16, 4, 10, seed=seed, aux=True)
        simg, saux, srays, states = r.render_snapshot(cam, 24, 16, 4, 10, seed=seed)
        assert simg.tobytes() == img.tobytes() and saux.tobytes() == aux.tobytes() and srays == rays
        arrays.update({f"s{seed}_image": img, f"s{seed}_aux": aux, f"s{seed}_rays": np.uint64(rays),
                       f"s{seed}_states": states})
    np.savez_compressed(os.path.join(HERE, "ref_material_renders.npz"), **arrays)


# (fixture name, reference.json scene, build_world arguments: scene id, model, crowd side, turn)
OBJ_SCENES = [("teapot", "teapot", 2, "models/teapot.obj", 20, 0.0),
              ("crowd", "crowd", 4, "models/teapot.obj", 8, 0.0),
              ("spot_crowd", "spot crowd", 4, "models/spot/spot.obj", 6, 150.0)]


def write_obj_scenes():
    """The reference's OBJ scenes, rebuilt from the fixture and checked equal
    to the reference's own description before writing."""
    sys.path.insert(0, os.path.dirname(HERE))
    import scene_fixture as sf
    from oracle.oracle import RefWorld
    for name, _, sid, model, side, turn in OBJ_SCENES:
        w = RefWorld(sid, os.path.join(REFERENCE, model), side, False, turn)
        f = sf.pack(w.desc, w.camera)
        a = abi.desc_arrays(w.desc)
        assert sf.triangles_of(f, "flat").tobytes() == a["triangles"].tobytes(), name
        for m in range(w.desc.n_meshes):
            assert sf.triangles_of(f, f"mesh{m}").tobytes() == a["meshes"][m].tobytes(), (name, m)
        trees = [(w.desc.flat_tree, "flat"), (w.desc.instance_tree, "instances")]
        trees += [(w.desc.meshes[m].tree, f"mesh{m}") for m in range(w.desc.n_meshes)]
        digests = {}
        for t, tname in trees:
            nodes = abi.view(t.nodes, t.n_nodes, abi.NODE_DTYPE)
            order = np.ctypeslib.as_array(t.order, (t.n_order,)).copy() if t.n_order else np.zeros(0, np.uint32)
            digests[tname] = [int(t.n_nodes), int(t.n_order),
                              hashlib.sha256(nodes.tobytes() + order.astype(np.uint32).tobytes()).hexdigest()]
        f["trees"] = np.array(json.dumps(digests))
        np.savez_compressed(os.path.join(HERE, f"ref_scene_{name}.npz"), **f)


def block_stats(images, block=20):
    """Per-seed image means (S x 3) and per-block means over seeds with their
    sigma (the reference's tests/render_test.py:96-133 statistics)."""
    means, blocks = [], []
    for img in images:
        h, w, _ = img.shape
        bw, bh = w // block, h // block
        b = img[:bh * block, :bw * block].reshape(bh, block, bw, block, 3).mean(axis=(1, 3), dtype=np.float64)
        blocks.append(b.reshape(-1))
        means.append(img.reshape(-1, 3).mean(axis=0, dtype=np.float64))
    blocks = np.array(blocks)
    return np.array(means), blocks.mean(axis=0), blocks.std(axis=0, ddof=1)


# (fixture name, generator, param, width, height, spp per seed)
CONVERGE = [("random_spheres", abi.PT_GEN_RANDOM_SPHERES, 0, 400, 225, 16),
            ("room_mesh", abi.PT_GEN_ROOM_MESH, 6, 1024, 1024, 64),
            ("instances", abi.PT_GEN_INSTANCES, 0, 1920, 1080, 32)]
CONVERGE_SEEDS = 16


def write_convergence():
    """Writes the convergence fixtures that are missing (delete one to write it again)."""
    threads = os.cpu_count() or 1
    for name, kind, param, w, h, spp in CONVERGE:
        if os.path.exists(os.path.join(HERE, f"ref_converge_{name}.npz")):
            continue
        g = pt.Generated(kind, seed=1, param=param)
        r = Reference(g.desc)
        images = []
        for k in range(CONVERGE_SEEDS):
            img, _, _ = r.render(g.camera, w, h, spp, 10, seed=1000 + k, threads=threads)
            images.append(img)
            print(f"\r{name}: {k + 1}/{CONVERGE_SEEDS} reference renders", end="", flush=True)
        print()
        means, bmean, bsigma = block_stats(images)
        np.savez_compressed(os.path.join(HERE, f"ref_converge_{name}.npz"), kind=kind, param=param, width=w, height=h,
                            spp=spp, seeds=np.arange(1000, 1000 + CONVERGE_SEEDS), image_means=means,
                            block_mean=bmean, block_sigma=bsigma, camera=np.frombuffer(bytes(g.camera), np.float32))


def write_blocks():
    ref_json = os.path.join(REFERENCE, "tests", "reference.json")
    with open(ref_json) as f:
        ref = json.load(f)
    blocks = {"width": ref["width"], "spp": ref["spp"], "block": ref["block"], "seeds": ref["seeds"]}
    arrays = {}
    scenes = [(s, s) for s in ("materials", "field", "room")] + [(n, s) for n, s, *_ in OBJ_SCENES]
    for key, scene in scenes:
        s = ref["scenes"][scene]
        arrays[f"{key}_blocks"] = np.array(s["blocks"], np.int32)
        arrays[f"{key}_mean"] = np.array(s["mean"], np.float64)
        arrays[f"{key}_sigma"] = np.array(s["sigma"], np.float64)
    np.savez_compressed(os.path.join(HERE, "reference_blocks.npz"), meta=json.dumps(blocks), **arrays)


def write_hits():
    for name, kind, param, (lo, hi), n in HIT_CASES:
        g = pt.Generated(kind, seed=1, param=param)
        r = Reference(g.desc)
        rays = pt.generate_rays(2024, lo, hi, n)
        # a few axis-aligned rays: zero direction components give infinite
        # inverses in the slab test
        rays[:6, 3:] = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1]], np.float32)
        hits, bad = r.trace_closest(rays)
        assert bad == 0, "re-composed hit disagrees with geometry::hit"
        occ = r.trace_any(rays)
        np.savez_compressed(os.path.join(HERE, f"ref_hits_{name}.npz"), rays=rays, hits=hits.view(np.uint32).reshape(-1, 6),
                            occluded=occ, kind=kind, param=param)


def write_renders():
    for name, kind, param, w, h, spp in RENDER_CASES:
        g = pt.Generated(kind, seed=1, param=param)
        r = Reference(g.desc)
        img, aux, rays, states = r.render_snapshot(g.camera, w, h, spp, 10, seed=5)
        cam = np.frombuffer(bytes(g.camera), np.float32)
        np.savez_compressed(os.path.join(HERE, f"ref_render_{name}.npz"), image=img, aux=aux, rays=np.uint64(rays),
                            states=states, camera=cam, kind=kind, param=param, width=w, height=h, spp=spp, seed=5)


def write_trees():
    digests = {}
    for name, kind, param in TREE_CASES:
        g = pt.Generated(kind, seed=1, param=param)
        r = Reference(g.desc)
        digests[name] = {"kind": kind, "param": param, "trees": tree_digest(reference_trees(r, g.desc))}
    with open(os.path.join(HERE, "ref_trees.json"), "w") as f:
        json.dump(digests, f, indent=1)


WRITERS = {"blocks": write_blocks, "hits": write_hits, "renders": write_renders, "trees": write_trees,
           "denoise": write_denoise, "edge": write_edge_hits, "materials": write_material_renders,
           "obj_scenes": write_obj_scenes, "converge": write_convergence}


def main():
    import argparse
    ap = argparse.ArgumentParser(description="writes the golden fixtures from the reference")
    ap.add_argument("--only", nargs="*", choices=sorted(WRITERS), help="write only these fixtures")
    args = ap.parse_args()
    for name in args.only or list(WRITERS):
        WRITERS[name]()
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
