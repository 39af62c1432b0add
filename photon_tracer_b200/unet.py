"""The learned denoiser: a U-Net over radiance, albedo, normal and depth
guides, trained on pairs of low- and high-spp renders (pt_unet_* and
pt_denoise_unet in include/photon_cuda.h). No reference counterpart: the
reference's denoiser is the a-trous filter (include/denoise.hpp), which is
this network's baseline.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Tuple

import numpy as np

from .abi import check, load

# (Cin, Cout, level, relu) of the 15 convolutions in forward order.
LAYERS: List[Tuple[int, int, int, bool]] = [
    (32, 32, 0, True), (32, 32, 0, True), (32, 64, 1, True), (64, 64, 1, True), (64, 96, 2, True),
    (96, 96, 2, True), (96, 128, 3, True), (128, 128, 3, True), (224, 96, 2, True), (96, 96, 2, True),
    (160, 64, 1, True), (64, 64, 1, True), (96, 32, 0, True), (32, 32, 0, True), (32, 16, 0, False)]
INPUT_CHANNELS = 10  # radiance 3, albedo 3, normal 3, depth 1


def param_layout():
    """(weight offset, (Cout, 3, 3, Cin), bias offset, Cout) per layer, and the total."""
    out, off = [], 0
    for cin, cout, _, _ in LAYERS:
        w = off
        off += cout * 9 * cin
        out.append((w, (cout, 3, 3, cin), off, cout))
        off += cout
    return out, off


def conv_flops(batch: int, height: int, width: int, algorithmic: bool = False) -> float:
    """Multiply-adds x 2 of the 15 convolutions at this size. By default the
    padding channels are included (they are computed: the first layer's 32
    input channels, the last layer's 16 outputs); algorithmic=True counts the
    network's own channels instead (10 inputs, 3 outputs)."""
    total = 0.0
    for k, (cin, cout, level, _) in enumerate(LAYERS):
        if algorithmic and k == 0:
            cin = INPUT_CHANNELS
        if algorithmic and k == len(LAYERS) - 1:
            cout = 3
        total += 2.0 * 9 * cin * cout * batch * (height >> level) * (width >> level)
    return total


class UNet:
    """A network on the current CUDA device. Tensors are torch CUDA float32."""

    def __init__(self, seed: int = 1):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.pt_unet_create(C.c_uint64(seed), C.byref(h)))
        self.h = h
        self.n_params = int(self.lib.pt_unet_num_params(h))

    def close(self) -> None:
        if self.h:
            self.lib.pt_unet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        check(self.lib.pt_unet_get_params(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        check(self.lib.pt_unet_set_params(self.h, p.ctypes.data_as(C.c_void_p)))

    def sync(self) -> None:
        """Waits for the current stream; raises if a tensor-core convolution timed out."""
        check(self.lib.pt_unet_sync(self.h, self._stream()))

    def tensor_cores(self, enable: bool) -> None:
        check(self.lib.pt_unet_set_tensor_cores(self.h, int(enable)))

    def save(self, path: str) -> None:
        np.save(path, self.params())

    def load(self, path: str) -> None:
        self.set_params(np.load(path))

    @staticmethod
    def _stream():
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def forward(self, x):
        """x: [B, H, W, 10] (radiance, albedo, normal, depth) -> [B, H, W, 3] radiance."""
        import torch
        B, H, W, c = x.shape
        assert c == INPUT_CHANNELS and x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()
        out = torch.empty((B, H, W, 3), dtype=torch.float32, device=x.device)
        check(self.lib.pt_unet_forward(self.h, B, H, W, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                                       self._stream()))
        return out

    def train_step(self, x, target, lr: float) -> float:
        B, H, W, _ = x.shape
        loss = C.c_float()
        check(self.lib.pt_unet_train_step(self.h, B, H, W, C.c_void_p(x.data_ptr()), C.c_void_p(target.data_ptr()),
                                          C.c_float(lr), C.byref(loss), self._stream()))
        return float(loss.value)

    def loss_grads(self, x, target):
        """(loss, parameter gradients, gradient w.r.t. the padded 32-channel input)."""
        import torch
        torch.cuda.synchronize()
        B, H, W, _ = x.shape
        loss = C.c_float()
        g = np.empty(self.n_params, np.float32)
        gi = np.empty((B, H, W, 32), np.float32)
        check(self.lib.pt_unet_loss_grads(self.h, B, H, W, C.c_void_p(x.data_ptr()), C.c_void_p(target.data_ptr()),
                                          C.byref(loss), g.ctypes.data_as(C.c_void_p),
                                          gi.ctypes.data_as(C.c_void_p)))
        return float(loss.value), g, gi

    def denoise(self, color, aux, depth):
        """One frame: color [H, W, 3], aux [H, W, 7] (the renderer's guides),
        depth [H, W] -> denoised [H, W, 3]."""
        import torch
        H, W, _ = color.shape
        out = torch.empty_like(color)
        check(self.lib.pt_denoise_unet(self.h, W, H, C.c_void_p(color.data_ptr()), C.c_void_p(aux.data_ptr()),
                                       C.c_void_p(depth.data_ptr()), C.c_void_p(out.data_ptr()), self._stream()))
        return out


def primary_depth(scene, cam, width: int, height: int):
    """Distance along each pixel's centre ray (pt_primary_depth_device), [H, W]."""
    import torch
    lib = load()
    out = torch.empty((height, width), dtype=torch.float32, device="cuda")
    check(lib.pt_primary_depth_device(scene.handle, C.byref(cam), width, height, C.c_void_p(out.data_ptr()),
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return out


def network_input(color, aux, depth):
    """The [H, W, 10] input of one frame from its colour, 7-float guides and depth."""
    import torch
    return torch.cat([color, aux[..., 0:6], depth[..., None]], dim=-1).contiguous()
