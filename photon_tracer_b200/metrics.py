"""Error metrics and the time-to-error study of the headline metric.

* relmse: mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2).
* ssim: structural similarity of luminance (Gaussian window sigma 1.5, 11 taps).
* GroundTruth: per-pixel radiance sums in FP64 over progressive passes on the
  GPU (pt_render_device with first_sample continuing the per-pixel sample
  numbering, pt_accumulate_pass adding each pass's averages * spp in double).
  save() / resume() checkpoint the sums, so a long ground truth (65,536 spp at
  1920x1080 is minutes per frame) can be built over several runs; a resumed
  run continues the sample numbers, so its sums equal an uninterrupted run's.
* time_to_error: the smallest power-of-two spp whose image reaches a relMSE
  target against ground truth, for plain path tracing and for path tracing
  followed by a denoiser (the a-trous filter or the learned U-Net), with the
  GPU time each took.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Callable, Optional

import numpy as np

from . import abi
from .abi import check, load


def relmse(x: np.ndarray, ref: np.ndarray, eps: float = 1e-2) -> float:
    x = np.asarray(x, np.float64)
    r = np.asarray(ref, np.float64)
    return float(np.mean((x - r) ** 2 / (r * r + eps)))


def _luminance(img: np.ndarray) -> np.ndarray:
    img = np.asarray(img, np.float64)
    return 0.2126 * img[..., 0] + 0.7152 * img[..., 1] + 0.0722 * img[..., 2]


def ssim(x: np.ndarray, ref: np.ndarray) -> float:
    """SSIM (Wang et al. 2004) on luminance mapped to display space
    (sqrt, clamped to [0, 1], the reference's gamma-2 display)."""
    from scipy.ndimage import gaussian_filter
    a = np.clip(np.sqrt(np.maximum(_luminance(x), 0)), 0, 1)
    b = np.clip(np.sqrt(np.maximum(_luminance(ref), 0)), 0, 1)
    k = dict(sigma=1.5, truncate=3.5)
    mu_a, mu_b = gaussian_filter(a, **k), gaussian_filter(b, **k)
    saa = gaussian_filter(a * a, **k) - mu_a ** 2
    sbb = gaussian_filter(b * b, **k) - mu_b ** 2
    sab = gaussian_filter(a * b, **k) - mu_a * mu_b
    c1, c2 = 0.01 ** 2, 0.03 ** 2
    s = ((2 * mu_a * mu_b + c1) * (2 * sab + c2)) / ((mu_a ** 2 + mu_b ** 2 + c1) * (saa + sbb + c2))
    return float(s.mean())


class GroundTruth:
    """FP64 per-pixel sums of a frame over progressive passes on the GPU."""

    def __init__(self, scene, cam, width: int, height: int, seed: int, max_bounces: int = 10, pass_spp: int = 256,
                 first_sample: int = 1 << 20):
        import torch
        self.scene, self.cam, self.w, self.h, self.seed = scene, cam, width, height, seed
        self.depth, self.pass_spp = max_bounces, pass_spp
        # Ground-truth samples are numbered from first_sample, away from the
        # sample numbers the renders under test use.
        self.first = first_sample
        self.spp = 0
        self.frame = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")
        self.sum = torch.zeros((height, width, 3), dtype=torch.float64, device="cuda")
        self.rays = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.stream = torch.cuda.current_stream().cuda_stream

    def add(self, passes: int) -> None:
        lib = load()
        for _ in range(passes):
            st = self.scene.settings(self.w, self.h, self.pass_spp, self.depth, self.seed, self.first + self.spp,
                                     abi.PT_MODE_MEGAKERNEL, abi.PT_RNG_SAMPLE)
            self.scene.render_device(self.cam, st, self.frame.data_ptr(), 0, self.rays.data_ptr(), self.stream)
            check(lib.pt_accumulate_pass(C.c_void_p(self.frame.data_ptr()), self.frame.numel(),
                                         float(self.pass_spp), C.c_void_p(self.sum.data_ptr()),
                                         C.c_void_p(self.stream)))
            self.spp += self.pass_spp
        self.scene.sync(self.stream)

    def image(self) -> np.ndarray:
        return (self.sum / self.spp).cpu().numpy()

    # What a checkpoint must agree on to continue the same sums.
    _KEYS = ("width", "height", "seed", "depth", "pass_spp", "first")

    def _fields(self) -> dict:
        return {"width": self.w, "height": self.h, "seed": self.seed, "depth": self.depth,
                "pass_spp": self.pass_spp, "first": self.first}

    def save(self, path: str, tag: str = "") -> None:
        """Writes the FP64 sums, the samples they hold and the frame they belong
        to (`tag` names the scene, e.g. "room:1001") to `path` (.npz), through a
        temporary file renamed into place."""
        tmp = path + ".tmp"
        with open(tmp, "wb") as f:
            np.savez(f, sum=self.sum.cpu().numpy(), spp=np.int64(self.spp), tag=np.str_(tag),
                     **{k: np.int64(v) for k, v in self._fields().items()})
        os.replace(tmp, path)

    def resume(self, path: str, tag: str = "") -> None:
        """Loads a checkpoint save() wrote for the same frame and scene; later
        add() calls continue its sample numbers. Raises ValueError when the
        checkpoint belongs to another frame, scene or sampling."""
        import torch
        with np.load(path, allow_pickle=False) as f:
            if str(f["tag"]) != tag:
                raise ValueError(f"{path}: checkpoint of scene {str(f['tag'])!r}, not {tag!r}")
            for k, mine in self._fields().items():
                if int(f[k]) != int(mine):
                    raise ValueError(f"{path}: checkpoint {k} = {int(f[k])}, this ground truth has {mine}")
            s = f["sum"]
            if s.dtype != np.float64 or s.shape != tuple(self.sum.shape):
                raise ValueError(f"{path}: sums of {s.dtype} {s.shape}, expected float64 {tuple(self.sum.shape)}")
            spp = int(f["spp"])
            if spp < 0 or spp % self.pass_spp:
                raise ValueError(f"{path}: {spp} samples is not a whole number of {self.pass_spp}-sample passes")
            if self.sum.is_cuda:  # nothing of this ground truth's may still be running on any stream
                torch.cuda.synchronize(self.sum.device)
            self.sum.copy_(torch.from_numpy(np.ascontiguousarray(s)))
            if self.sum.is_cuda:
                torch.cuda.synchronize(self.sum.device)
            self.spp = spp


def _timed(fn: Callable[[], None]) -> float:
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    fn()
    b.record()
    torch.cuda.synchronize()
    return float(a.elapsed_time(b))


def render_and_denoise(scene, cam, width, height, spp, seed, max_bounces=10):
    """A frame with its guides, then the a-trous filter, all on the device.
    Returns (noisy image, denoised image, GPU ms of render + filter)."""
    import torch
    lib = load()
    out = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")
    aux = torch.empty((height, width, 7), dtype=torch.float32, device="cuda")
    den = torch.empty_like(out)
    scratch = torch.empty(lib.pt_denoise_atrous_scratch_floats(width, height), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = scene.settings(width, height, spp, max_bounces, seed, 0, abi.PT_MODE_MEGAKERNEL, abi.PT_RNG_SAMPLE)
    guides = {}

    def run():
        scene.render_device(cam, st, out.data_ptr(), aux.data_ptr(), 0, stream)
        # the guides the reference's CLI derives (src/main.cpp:176-183)
        albedo = aux[..., 0:3].contiguous()
        normal = aux[..., 3:6].contiguous()
        lum = 0.2126 * out[..., 0] + 0.7152 * out[..., 1] + 0.0722 * out[..., 2]
        variance = ((aux[..., 6] - lum * lum) / spp).contiguous()
        guides["keep"] = (albedo, normal, variance)
        check(lib.pt_denoise_atrous_device(width, height, C.c_void_p(out.data_ptr()), C.c_void_p(albedo.data_ptr()),
                                           C.c_void_p(normal.data_ptr()), C.c_void_p(variance.data_ptr()),
                                           C.c_void_p(den.data_ptr()), C.c_void_p(scratch.data_ptr()),
                                           C.c_void_p(stream)))
    ms = _timed(run)
    scene.sync(stream)
    return out.cpu().numpy(), den.cpu().numpy(), ms


def render_and_unet(net, scene, cam, width, height, spp, seed, max_bounces=10):
    """A frame with its guides and depth, then the learned denoiser, all on the
    device. Returns (noisy image, denoised image, GPU ms of render + depth + network)."""
    from .denoiser import denoise_frame
    res = {}

    def run():
        res["noisy"], res["den"] = denoise_frame(net, scene, cam, width, height, spp, seed, max_bounces)
    ms = _timed(run)
    scene.sync(torch_stream())
    net.sync()
    return res["noisy"].cpu().numpy(), res["den"].cpu().numpy(), ms


def torch_stream() -> int:
    import torch
    return torch.cuda.current_stream().cuda_stream


def time_to_error(scene, cam, width: int, height: int, truth: np.ndarray, seed: int = 7, target: float = 0.01,
                  max_spp: int = 4096, denoise: Optional[str] = None, max_bounces: int = 10, net=None) -> dict:
    """The smallest power-of-two spp reaching relMSE <= target, and its GPU time.
    denoise None: plain path tracing; "atrous": followed by the a-trous filter;
    "unet": followed by the learned denoiser `net`."""
    import torch
    out = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # One untimed pass first: the denoisers allocate their workspaces for a
    # frame size on first use.
    if denoise == "unet":
        render_and_unet(net, scene, cam, width, height, 1, seed + 1, max_bounces)
    elif denoise is not None:
        render_and_denoise(scene, cam, width, height, 1, seed + 1, max_bounces)
    history = []
    spp = 1
    while spp <= max_spp:
        if denoise is None:
            st = scene.settings(width, height, spp, max_bounces, seed, 0, abi.PT_MODE_MEGAKERNEL, abi.PT_RNG_SAMPLE)
            ms = _timed(lambda: scene.render_device(cam, st, out.data_ptr(), 0, 0, stream))
            scene.sync(stream)
            img = out.cpu().numpy()
        elif denoise == "unet":
            _, img, ms = render_and_unet(net, scene, cam, width, height, spp, seed, max_bounces)
        else:
            _, img, ms = render_and_denoise(scene, cam, width, height, spp, seed, max_bounces)
        err = relmse(img, truth)
        history.append({"spp": spp, "ms": round(ms, 3), "relmse": err, "ssim": ssim(img, truth)})
        if err <= target:
            return {"reached": True, "spp": spp, "ms": ms, "relmse": err, "history": history}
        spp *= 2
    return {"reached": False, "spp": None, "ms": None, "relmse": history[-1]["relmse"], "history": history}
