"""CPU float64 reference of the U-Net in vdropimpact_b200/csrc/unet.cu, for
the numerics tests of its tensor-core kernels.

forward() restates the network layer by layer with torch's float64 conv2d on
the CPU. With bf16=True it rounds to bfloat16 (round to nearest even) at the
points where the CUDA kernels store BF16: the weights, the packed input, every
hidden activation and a pooled convolution input. The rounding is a
straight-through operation (value rounded, derivative one). The backward
also rounds each convolution's output gradient to BF16, as the CUDA backward
does before its two GEMMs, so autograd restates the CUDA backward up to FP32
accumulation order.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

# {cin, cout, mode (0 direct, 1 nearest up x2, 2 mean pool 2x2), relu, skip, src}
SPEC = [(16, 16, 0, 1, -1, -1), (16, 16, 0, 1, -1, 0), (16, 32, 2, 1, -1, 1), (32, 32, 0, 1, -1, 2),
        (32, 64, 2, 1, -1, 3), (64, 64, 0, 1, -1, 4), (64, 64, 2, 1, -1, 5), (64, 64, 0, 1, -1, 6),
        (64, 64, 1, 1, 5, 7), (64, 32, 0, 1, -1, 8), (32, 32, 1, 1, 3, 9), (32, 16, 0, 1, -1, 10),
        (16, 16, 1, 1, 1, 11), (16, 16, 0, 0, -1, 12)]


def param_count() -> int:
    return sum(9 * ci * co + co for ci, co, *_ in SPEC)


def split_params(flat: np.ndarray):
    """Per layer (w [9][cout][cin], b [cout]) from the flat layout of
    vdi_unet_params."""
    out, off = [], 0
    for ci, co, *_ in SPEC:
        nw = 9 * ci * co
        out.append((flat[off:off + nw].reshape(9, co, ci), flat[off + nw:off + nw + co]))
        off += nw + co
    assert off == flat.size
    return out


def _bf16(x, on: bool):
    if not on:
        return x
    return x + (x.to(torch.bfloat16).to(x.dtype) - x).detach()


class _GradToBF16(torch.autograd.Function):
    """Identity whose backward rounds the incoming gradient to bfloat16: the
    CUDA backward stores the output gradient of a convolution as BF16 GEMM
    operands (weight gradient and input gradient alike)."""

    @staticmethod
    def forward(ctx, x):
        return x.view_as(x)

    @staticmethod
    def backward(ctx, g):
        return g.to(torch.bfloat16).to(g.dtype)


def forward(params, x, *, bf16: bool = True, requires_grad: bool = False):
    """x: (B, H, W) array. Returns (y (B, H, W) float64 tensor, weights) with
    weights the list of float64 weight tensors [9][cout][cin] (leaves with
    gradients when requires_grad)."""
    x = torch.as_tensor(np.asarray(x), dtype=torch.float64)
    B, H, W = x.shape
    inp = torch.zeros(B, 16, H, W, dtype=torch.float64)
    inp[:, 0] = x
    inp = _bf16(inp, bf16)
    ws = []
    acts = []
    for k, ((ci, co, mode, relu, skip, src), (w, b)) in enumerate(zip(SPEC, params)):
        wt = torch.tensor(np.asarray(w, dtype=np.float64), requires_grad=requires_grad)
        ws.append(wt)
        bt = torch.as_tensor(np.asarray(b, dtype=np.float64))
        s = inp if src < 0 else acts[src]
        if mode == 1:
            s = s.repeat_interleave(2, dim=2).repeat_interleave(2, dim=3)
        elif mode == 2:
            s = _bf16(F.avg_pool2d(s, 2), bf16)
        # weight [co][ci][ky][kx] from [tap = 3 ky + kx][co][ci]
        kern = _bf16(wt, bf16).reshape(3, 3, co, ci).permute(2, 3, 0, 1)
        y = F.conv2d(s, kern, padding=1)
        if bf16:
            y = _GradToBF16.apply(y)
        y = y + bt.view(1, -1, 1, 1)
        if skip >= 0:
            y = y + acts[skip]
        if relu:
            y = torch.relu(y)
        if k < len(SPEC) - 1:
            y = _bf16(y, bf16)
        acts.append(y)
    return acts[-1][:, 0], ws


def loss_and_grads(params, x, t, *, bf16: bool = True):
    """Loss mean((y - t)^2) and the weight gradients [9][cout][cin] of every
    layer (numpy float64)."""
    y, ws = forward(params, x, bf16=bf16, requires_grad=True)
    tt = torch.as_tensor(np.asarray(t), dtype=torch.float64)
    loss = torch.mean((y - tt) ** 2)
    loss.backward()
    return float(loss.detach()), [w.grad.numpy() for w in ws]
