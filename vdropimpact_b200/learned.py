"""Learned initial guess for the MAC projection solve.

The multigrid solve of A q = b starts from a time-extrapolated guess z0. Its
error e = q - z0 satisfies A e = r with r = b - A z0, so a network trained on
(r, e) pairs learns an approximate inverse of A on the residuals the
simulation produces. UNet binds the network of include/vdi.h (BF16 tensor-core
kernels, FP32 accumulation, Adam); harvest() collects pairs from a running
simulation; train() fits the network on the GPU; Fluid2D.attach_unet() makes
it the VDI_GUESS_LEARNED guess. The multigrid always iterates to tolerance
from the corrected guess, so the network changes the V-cycle count, not the
converged result.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import check, lib


def _torch():
    import torch
    return torch


class UNet:
    """The U-Net on an H x W grid (H a multiple of 8, W of 16)."""

    def __init__(self, H: int, W: int, batch: int = 8, seed: int = 1, stream=None):
        self.H, self.W, self.batch = H, W, batch
        h = C.c_void_p()
        s = None if stream is None else C.c_void_p(int(getattr(stream, "cuda_stream", stream)))
        check(lib().vdi_unet_create(H, W, batch, seed, s, C.byref(h)), "vdi_unet_create")
        self._h = h
        self.out_scale = 1.0

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                lib().vdi_unet_destroy(self._h)
                self._h = None
        except Exception:
            pass

    @property
    def param_count(self) -> int:
        return int(lib().vdi_unet_param_count(self._h))

    def forward(self, x):
        """x: float32 CUDA tensor (B, H, W) -> (B, H, W)."""
        torch = _torch()
        x = x.contiguous()
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        check(lib().vdi_unet_forward(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.shape[0]),
              "vdi_unet_forward")
        torch.cuda.synchronize()
        return y

    def train_step(self, x, t, lr: float) -> float:
        torch = _torch()
        loss = C.c_float()
        x = x.contiguous()
        t = t.contiguous()
        torch.cuda.synchronize()
        check(lib().vdi_unet_train_step(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()), x.shape[0],
                                        lr, C.byref(loss)), "vdi_unet_train_step")
        return loss.value

    def gradients(self, x, t, layer: int, shape):
        torch = _torch()
        g = np.zeros(int(np.prod(shape)), dtype=np.float32)
        loss = C.c_float()
        torch.cuda.synchronize()
        check(lib().vdi_unet_gradients(self._h, C.c_void_p(x.contiguous().data_ptr()),
                                       C.c_void_p(t.contiguous().data_ptr()), x.shape[0], layer,
                                       g.ctypes.data_as(C.c_void_p), C.byref(loss)), "vdi_unet_gradients")
        return g.reshape(shape), loss.value

    def get_params(self) -> np.ndarray:
        buf = np.zeros(self.param_count, dtype=np.float32)
        check(lib().vdi_unet_params(self._h, buf.ctypes.data_as(C.c_void_p), buf.size, 0), "vdi_unet_params")
        return buf

    def set_params(self, buf: np.ndarray):
        buf = np.ascontiguousarray(buf, dtype=np.float32)
        check(lib().vdi_unet_params(self._h, buf.ctypes.data_as(C.c_void_p), buf.size, 1), "vdi_unet_params")


def _restrict(a, m, n, f):
    torch = _torch()
    return a.view(n // f, f, m // f, f).mean(dim=(1, 3))


def harvest(sim, steps: int, dt: float, factor: int, mac):
    """Runs `steps` steps of sim (quadratic-extrapolation guess) and returns
    (inputs, targets): the RMS-normalised restricted residuals of the
    extrapolated guess and the restricted errors scaled by xxsp / rms, as
    float32 CUDA tensors (N, n/f, m/f). mac is an MgsMac with the sim's grid,
    used for A z."""
    torch = _torch()
    m, n = sim.m, sim.n
    xxsp = 1.0 / (sim.dx * sim.dx)
    pb, nb_ = sim.device_field(6)
    pq, _ = sim.device_field(7)
    b_dev = _wrap(torch, pb, nb_)
    q_dev = _wrap(torch, pq, nb_)
    hist = []
    xs, ts = [], []
    for k in range(steps):
        sim.step_forward(dt, 1)
        sim.synchronize()
        q = q_dev.clone()
        b = b_dev.clone()
        if len(hist) == 3:
            z0 = 3 * hist[2] - 3 * hist[1] + hist[0]
            r = b - mac.apply(z0)
            e = q - z0
            rms = float(torch.sqrt(torch.mean(r * r)))
            if rms > 0:
                xs.append((_restrict(r.view(n, m), m, n, factor) / rms).float())
                ts.append((_restrict(e.view(n, m), m, n, factor) * (xxsp / rms)).float())
        hist = (hist + [q])[-3:]
    return torch.stack(xs), torch.stack(ts)


def train(net: UNet, xs, ts, iters: int = 2000, lr: float = 1e-3, batch: int = 4, seed: int = 0, log=None):
    """Fits net to (xs, ts) with Adam; the targets are divided by a global
    scale (stored in net.out_scale) so that they are of order one."""
    torch = _torch()
    scale = float(torch.sqrt(torch.mean(ts * ts)))
    net.out_scale = scale
    tn = ts / scale
    g = torch.Generator(device="cpu").manual_seed(seed)
    losses = []
    N = xs.shape[0]
    for it in range(iters):
        idx = torch.randint(0, N, (batch,), generator=g).to(xs.device)
        l = net.train_step(xs[idx], tn[idx], lr if it < iters * 3 // 4 else lr * 0.1)
        losses.append(l)
        if log and it % 200 == 0:
            log(it, l)
    return losses


def _wrap(torch, ptr, n):
    class _Iface:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                             "version": 3, "strides": None}
    return torch.as_tensor(_Iface(), device="cuda")
