"""Plain PyTorch fp32 restatement of the U-Net denoiser (checker for the CUDA
network, test infrastructure only). It rounds to bfloat16 where the CUDA
network stores bfloat16 (the network input, the weights used by every
convolution, and every activation but the last) and is fp32 elsewhere; the
rounding is straight-through, so gradients flow in fp32 like the CUDA
backward's."""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

from photon_tracer_b200.unet import LAYERS, param_layout


def bf16(x: torch.Tensor) -> torch.Tensor:
    return x + (x.to(torch.bfloat16).to(torch.float32) - x).detach()


def unpack(params: np.ndarray):
    """Per layer (weight [Cout, Cin, 3, 3] as an NCHW conv weight, bias) leaf tensors."""
    layout, total = param_layout()
    assert params.size == total
    out = []
    for w_off, (co, kh, kw, ci), b_off, _ in layout:
        w = params[w_off:w_off + co * kh * kw * ci].reshape(co, kh, kw, ci).transpose(0, 3, 1, 2)
        b = params[b_off:b_off + co]
        out.append((torch.tensor(np.ascontiguousarray(w), requires_grad=True),
                    torch.tensor(b.copy(), requires_grad=True)))
    return out


def pack_grads(weights) -> np.ndarray:
    layout, total = param_layout()
    g = np.zeros(total, np.float32)
    for (w_off, (co, kh, kw, ci), b_off, _), (w, b) in zip(layout, weights):
        g[w_off:w_off + co * kh * kw * ci] = w.grad.detach().numpy().transpose(0, 2, 3, 1).reshape(-1)
        g[b_off:b_off + co] = b.grad.detach().numpy()
    return g


def network_input(x: torch.Tensor) -> torch.Tensor:
    """[B, H, W, 10] float guides -> [B, 32, H, W] the padded input."""
    rad = torch.log1p(torch.clamp(x[..., 0:3], min=0))
    depth = torch.log1p(torch.clamp(x[..., 9:10], min=0))
    z = torch.zeros(x.shape[:-1] + (22,), dtype=x.dtype)
    t = torch.cat([rad, x[..., 3:9], depth, z], dim=-1)
    return t.permute(0, 3, 1, 2).contiguous()


def forward(weights, inp: torch.Tensor) -> torch.Tensor:
    """inp [B, 32, H, W] (already bf16-valued) -> [B, 16, H, W] log radiance (fp32)."""
    def conv(i, x):
        w, b = weights[i]
        y = F.conv2d(x, bf16(w), b, padding=1)
        if LAYERS[i][3]:
            return bf16(F.relu(y))
        return y

    up = lambda x: F.interpolate(x, scale_factor=2, mode="nearest")
    a1 = conv(1, conv(0, inp))
    a3 = conv(3, conv(2, F.max_pool2d(a1, 2)))
    a5 = conv(5, conv(4, F.max_pool2d(a3, 2)))
    a7 = conv(7, conv(6, F.max_pool2d(a5, 2)))
    d2 = conv(9, conv(8, torch.cat([up(a7), a5], 1)))
    d1 = conv(11, conv(10, torch.cat([up(d2), a3], 1)))
    d0 = conv(13, conv(12, torch.cat([up(d1), a1], 1)))
    return conv(14, d0)


def loss_and_grads(params: np.ndarray, x: np.ndarray, target: np.ndarray):
    """(loss, parameter gradients, input gradient [B, H, W, 32], output [B, H, W, 3])
    of the mean L1 distance of log radiance, all on the CPU in fp32."""
    weights = unpack(params)
    xi = bf16(network_input(torch.tensor(x))).detach().requires_grad_(True)
    pred = forward(weights, xi)
    tgt = torch.log1p(torch.clamp(torch.tensor(target), min=0)).permute(0, 3, 1, 2)
    loss = (pred[:, 0:3] - tgt).abs().mean()
    loss.backward()
    out = torch.clamp(torch.expm1(pred[:, 0:3]), min=0).permute(0, 2, 3, 1)
    return (loss.item(), pack_grads(weights), xi.grad.permute(0, 2, 3, 1).numpy(), out.detach().numpy())
