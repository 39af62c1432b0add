"""Training and use of the learned denoiser on frames this tracer renders.

* Training set: procedural scenes from fresh seeds of the random-spheres,
  room-mesh and instancing generators, seen through jittered cameras and
  through each generator's own camera, rendered at low spp (inputs, several
  spp levels so the network meets every noise level it is used at) and at
  high spp with other sample numbers (targets). Inputs carry the renderer's albedo and normal guides and the
  primary-ray depth.
* Training: random crops, Adam on the mean L1 distance of log radiance
  (pt_unet_train_step, the library's own forward and backward kernels).
* Use: render + depth guide + pt_denoise_unet, all on the device.

Command line (writes the weights as bfloat16 bits, the precision the network
computes in):
    python -m photon_tracer_b200.denoiser train --out weights.npy
"""
from __future__ import annotations

import argparse
import json
import os
import time
from typing import Dict, List

import numpy as np

from . import abi
from .api import Generated, Scene, camera_look_at
from .unet import UNet, conv_flops, primary_depth

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "unet_bf16.npy")

# kind -> (generator, lookfrom, lookat, vfov, camera jitter scale)
SCENES = {
    "spheres": (abi.PT_GEN_RANDOM_SPHERES, (13.0, 2.0, 3.0), (0.0, 0.0, 0.0), 20.0, 1.5),
    "room": (abi.PT_GEN_ROOM_MESH, (0.0, 0.0, 3.3), (0.0, 0.0, 0.0), 40.0, 0.25),
    "instances": (abi.PT_GEN_INSTANCES, (0.0, 35.0, 140.0), (0.0, 0.0, 0.0), 45.0, 12.0),
}
INPUT_SPP = (1, 2, 4, 8, 16, 32)
TARGET_FIRST_SAMPLE = 1 << 22  # target samples are numbered apart from the inputs'


def _stream() -> int:
    import torch
    return torch.cuda.current_stream().cuda_stream


def render(scene: Scene, cam, width: int, height: int, spp: int, seed: int, first_sample: int = 0,
           aux: bool = True, max_bounces: int = 10):
    """(colour [H, W, 3], guides [H, W, 7] or None) on the device."""
    import torch
    out = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")
    ax = torch.empty((height, width, 7), dtype=torch.float32, device="cuda") if aux else None
    st = Scene.settings(width, height, spp, max_bounces, seed, first_sample, abi.PT_MODE_MEGAKERNEL,
                        abi.PT_RNG_SAMPLE)
    scene.render_device(cam, st, out.data_ptr(), ax.data_ptr() if aux else 0, 0, _stream())
    return out, ax


def network_input(color, aux, depth):
    import torch
    return torch.cat([color, aux[..., 0:6], depth[..., None]], dim=-1)


def scene_and_camera(kind: str, seed: int, aspect: float, jitter: bool):
    gen, frm, at, vfov, scale = SCENES[kind]
    g = Generated(gen, seed=seed)
    frm, at = np.array(frm), np.array(at)
    if jitter:
        rng = np.random.default_rng(seed * 7919 + 17)
        frm = frm + rng.normal(0, scale, 3) * np.array([1.0, 0.4, 1.0])
        at = at + rng.normal(0, scale * 0.15, 3)
        vfov = vfov * float(rng.uniform(0.75, 1.25))
    cam = camera_look_at(tuple(frm), tuple(at), vfov, aspect)
    return g, Scene(g), cam


def render_pair(kind: str, seed: int, width: int, height: int, target_spp: int, jitter: bool) -> Dict:
    """One training frame: inputs at every INPUT_SPP level and the target, on the device."""
    g, scene, cam = scene_and_camera(kind, seed, width / height, jitter=jitter)
    return render_view(scene, cam, kind, seed, width, height, target_spp)


def render_view(scene: Scene, cam, kind: str, seed: int, width: int, height: int, target_spp: int) -> Dict:
    """Inputs at every INPUT_SPP level and the target of one view of a scene, on the device."""
    import torch
    depth = primary_depth(scene, cam, width, height)
    inputs = []
    for spp in INPUT_SPP:
        c, a = render(scene, cam, width, height, spp, seed, first_sample=0)
        inputs.append(network_input(c, a, depth))
    target, _ = render(scene, cam, width, height, target_spp, seed, first_sample=TARGET_FIRST_SAMPLE, aux=False)
    scene.sync(_stream())
    return {"inputs": torch.stack(inputs).contiguous(), "target": target, "kind": kind, "seed": seed}


def make_crop_set(kind: str, crops: int, size: int, target_spp: int, seed0: int, views_per_scene: int,
                  tiles: int = 2, log=print) -> List[Dict]:
    """`crops` square crops of `size` of the generator `kind`: scenes from
    seeds seed0, seed0 + 1, .., each seen through views_per_scene jittered
    cameras (each view's own seed drives its camera and its samples); each
    view is rendered at (tiles * size)^2 and cut into tiles^2 crops, because
    a frame with fewer pixels than the megakernel has lanes leaves lanes idle
    (every lane renders a whole pixel's samples)."""
    data = []
    seed = seed0
    while len(data) < crops:
        g = Generated(SCENES[kind][0], seed=seed)
        scene = Scene(g)
        for v in range(views_per_scene):
            if len(data) >= crops:
                break
            view_seed = seed * 16 + v
            _, frm, at, vfov, scale = SCENES[kind]
            rng = np.random.default_rng(view_seed * 7919 + 17)
            f = np.array(frm) + rng.normal(0, scale, 3) * np.array([1.0, 0.4, 1.0])
            a = np.array(at) + rng.normal(0, scale * 0.15, 3)
            cam = camera_look_at(tuple(f), tuple(a), vfov * float(rng.uniform(0.75, 1.25)), 1.0)
            t0 = time.perf_counter()
            full = render_view(scene, cam, kind, view_seed, tiles * size, tiles * size, target_spp)
            for ty in range(tiles):
                for tx in range(tiles):
                    if len(data) >= crops:
                        break
                    ys, xs = slice(ty * size, (ty + 1) * size), slice(tx * size, (tx + 1) * size)
                    data.append({"inputs": full["inputs"][:, ys, xs].contiguous(),
                                 "target": full["target"][ys, xs].contiguous(), "kind": kind, "seed": view_seed})
            del full
            log(f"view {kind} scene {seed} view {v}: {time.perf_counter() - t0:.2f} s")
        scene.close()
        seed += 1
    return data


def make_training_set(frames_per_kind: int, size: int, target_spp: int, seed0: int = 100,
                      kinds=("spheres", "room", "instances"), default_frames: int = 0, log=print) -> List[Dict]:
    """Per frame: 'inputs' [len(INPUT_SPP), H, W, 10] and 'target' [H, W, 3] on the device.
    frames_per_kind square frames of `size` through jittered cameras (seeds
    seed0 + 1000 k + f), and default_frames 640x360 frames through each
    generator's own camera (seeds seed0 + 1000 k + 500 + f)."""
    data = []
    for k, kind in enumerate(kinds):
        jobs = [(seed0 + 1000 * k + f, size, size, True) for f in range(frames_per_kind)]
        jobs += [(seed0 + 1000 * k + 500 + f, 640, 360, False) for f in range(default_frames)]
        for seed, w, h, jitter in jobs:
            t0 = time.perf_counter()
            data.append(render_pair(kind, seed, w, h, target_spp, jitter))
            log(f"frame {kind} seed {seed} {w}x{h}: {time.perf_counter() - t0:.2f} s")
    return data


def sample_batch(data, rng, batch: int, crop: int):
    import torch
    xs, ts = [], []
    for _ in range(batch):
        d = data[int(rng.integers(len(data)))]
        L, H, W, _ = d["inputs"].shape
        lvl = int(rng.integers(L))
        y, x = int(rng.integers(H - crop + 1)), int(rng.integers(W - crop + 1))
        xs.append(d["inputs"][lvl, y:y + crop, x:x + crop])
        ts.append(d["target"][y:y + crop, x:x + crop])
    return torch.stack(xs).contiguous(), torch.stack(ts).contiguous()


def train(net: UNet, data, steps: int, batch: int = 8, crop: int = 128, lr: float = 1e-3, seed: int = 0,
          max_seconds: float = float("inf"), log=print) -> List[float]:
    """Adam at lr for the first 80% of the steps, then lr/10; stops early
    after max_seconds (the step count then shrinks to what ran)."""
    rng = np.random.default_rng(seed)
    losses = []
    t0 = time.perf_counter()
    for s in range(steps):
        if time.perf_counter() - t0 > max_seconds:
            log(f"stopped after {s} steps (time limit)")
            break
        x, t = sample_batch(data, rng, batch, crop)
        losses.append(net.train_step(x, t, lr if s < 0.8 * steps else lr * 0.1))
        if (s + 1) % max(1, steps // 20) == 0:
            log(f"step {s + 1}/{steps}: loss {np.mean(losses[-50:]):.4f} ({time.perf_counter() - t0:.1f} s)")
    return losses


def save_bf16(params: np.ndarray, path: str) -> None:
    """float32 -> bfloat16 bits (round to nearest even), as uint16."""
    u = np.ascontiguousarray(params, np.float32).view(np.uint32)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.save(path, r)


def load_bf16(path: str) -> np.ndarray:
    return (np.load(path).astype(np.uint32) << 16).view(np.float32)


def trained(path: str = WEIGHTS) -> UNet:
    """A network with the committed trained weights."""
    if not os.path.exists(path):
        raise FileNotFoundError(f"no trained denoiser weights at {path}")
    net = UNet(seed=0)
    net.set_params(load_bf16(path))
    return net


def denoise_frame(net: UNet, scene: Scene, cam, width: int, height: int, spp: int, seed: int, max_bounces: int = 10):
    """Render with guides, depth guide, network -- all enqueued on the current stream."""
    color, aux = render(scene, cam, width, height, spp, seed, max_bounces=max_bounces)
    depth = primary_depth(scene, cam, width, height)
    return color, net.denoise(color, aux, depth)


def time_forward(net: UNet, width: int = 1920, height: int = 1080, reps: int = 10) -> Dict:
    """GPU time of the network at one frame size, tensor cores on and off."""
    import torch
    color = torch.rand((height, width, 3), device="cuda")
    aux = torch.rand((height, width, 7), device="cuda")
    depth = torch.rand((height, width), device="cuda")
    out = {}
    for tc in (True, False):
        net.tensor_cores(tc)
        for _ in range(2):
            net.denoise(color, aux, depth)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n = reps if tc else max(1, reps // 5)
        torch.cuda.synchronize()
        a.record()
        for _ in range(n):
            net.denoise(color, aux, depth)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / n
        hp, wp = (height + 7) // 8 * 8, (width + 7) // 8 * 8
        out["tensor_cores" if tc else "cuda_cores"] = {"ms": round(ms, 3),
                                                       "tflops": round(conv_flops(1, hp, wp) / ms / 1e9, 1)}
    net.tensor_cores(True)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="train the learned denoiser on frames this tracer renders")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", required=True)
    t.add_argument("--frames", type=int, default=16, help="jittered square frames per scene kind")
    t.add_argument("--default-frames", type=int, default=0, help="640x360 frames per kind through its own camera")
    t.add_argument("--size", type=int, default=384)
    t.add_argument("--target-spp", type=int, default=1024)
    t.add_argument("--steps", type=int, default=3000)
    t.add_argument("--batch", type=int, default=8)
    t.add_argument("--crop", type=int, default=128)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--init", default=None, help="start from these weights")
    t.add_argument("--max-minutes", type=float, default=float("inf"), help="stop training after this long")
    t.add_argument("--mix", nargs="+", default=None, metavar="KIND:FRAMES:DEFAULT:SEED0",
                   help="per-kind training frames instead of --frames/--default-frames for all kinds: "
                        "square frames from seeds SEED0.., default-camera frames from SEED0+500..")
    t.add_argument("--train-seed", type=int, default=0, help="seed of the crop sampler")
    t.add_argument("--crops", nargs="+", default=None, metavar="KIND:COUNT:SEED0",
                   help="square crops of --size per kind instead of --mix / --frames: scenes from seeds SEED0.., "
                        "--views-per-scene jittered views each, every view rendered at (--tiles * --size)^2 and cut "
                        "into --tiles^2 crops")
    t.add_argument("--views-per-scene", type=int, default=1)
    t.add_argument("--tiles", type=int, default=2)
    p = sub.add_parser("time")
    p.add_argument("--width", type=int, default=1920)
    p.add_argument("--height", type=int, default=1080)
    f = sub.add_parser("frames", help="denoise seeded random frames with the trained weights (a profiling driver)")
    f.add_argument("--count", type=int, default=3)
    f.add_argument("--width", type=int, default=1920)
    f.add_argument("--height", type=int, default=1080)
    args = ap.parse_args(argv)
    import torch
    torch.cuda.init()
    if args.cmd == "time":
        print(json.dumps(time_forward(UNet(seed=1), args.width, args.height)))
        return 0
    if args.cmd == "frames":
        net = trained()
        g = torch.Generator(device="cuda").manual_seed(1)
        color = torch.rand((args.height, args.width, 3), device="cuda", generator=g)
        aux = torch.rand((args.height, args.width, 7), device="cuda", generator=g)
        depth = torch.rand((args.height, args.width), device="cuda", generator=g)
        for _ in range(args.count):
            net.denoise(color, aux, depth)
        net.sync()
        return 0
    t0 = time.perf_counter()
    if args.crops:
        data = []
        for spec in args.crops:
            kind, count, seed0 = spec.split(":")
            data += make_crop_set(kind, int(count), args.size, args.target_spp, int(seed0), args.views_per_scene,
                                  args.tiles)
    elif args.mix:
        data = []
        for spec in args.mix:
            kind, frames, default, seed0 = spec.split(":")
            data += make_training_set(int(frames), args.size, args.target_spp, seed0=int(seed0), kinds=(kind,),
                                      default_frames=int(default))
    else:
        data = make_training_set(args.frames, args.size, args.target_spp, default_frames=args.default_frames)
    t_data = time.perf_counter() - t0
    net = UNet(seed=1)
    if args.init:
        net.set_params(load_bf16(args.init))
    t0 = time.perf_counter()
    losses = train(net, data, args.steps, args.batch, args.crop, args.lr, seed=args.train_seed,
                   max_seconds=60 * args.max_minutes)
    t_train = time.perf_counter() - t0
    save_bf16(net.params(), args.out)
    np.save(os.path.splitext(args.out)[0] + "_losses.npy", np.array(losses, np.float32))
    print(json.dumps({"frames": len(data), "data_s": round(t_data, 1), "train_s": round(t_train, 1),
                      "steps": len(losses), "final_loss": float(np.mean(losses[-100:])),
                      "ms_per_step": round(1000 * t_train / max(1, len(losses)), 2)}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
