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

    def guess(self, mac, factor: int):
        """Adds the network's correction to mac.z (the residual of the
        current mac.z against mac.b is its input): the learned initial guess
        of a standalone MAC solve (vdi_unet_guess)."""
        torch = _torch()
        xxsp = mac.xxsp
        torch.cuda.synchronize()
        check(lib().vdi_unet_guess(self._h, mac._h, factor, float(self.out_scale) / xxsp,
                                   C.c_void_p(mac.b.data_ptr()), C.c_void_p(mac.z.data_ptr())), "vdi_unet_guess")


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


# ---------------------------------------------------------------------------
# The learned guess on the single-projection workload: solves from scratch
# (zero initial guess), where the network's prediction of the solution is
# the whole initial guess.

def gaussian_sources(m: int, n: int, seeds, count: int = 64):
    """The sources of projection_source (the zero-mean sum of `count`
    Gaussians with parameters drawn from numpy's generator seeded with each
    seed, in the same order) for many seeds, evaluated on the GPU as outer
    products: float64 CUDA tensor (len(seeds), n*m)."""
    torch = _torch()
    dev = "cuda"
    x = (torch.arange(m, dtype=torch.float64, device=dev) + 0.5) / m
    y = (torch.arange(n, dtype=torch.float64, device=dev) + 0.5) / n * (n / m)
    out = torch.empty(len(seeds), n * m, dtype=torch.float64, device=dev)
    for k, sd in enumerate(seeds):
        rng = np.random.default_rng(sd)
        prm = np.empty((count, 4))
        for q in range(count):
            prm[q] = (rng.uniform(0, 1), rng.uniform(0, n / m), rng.uniform(0.01, 0.1), rng.standard_normal())
        P = torch.from_numpy(prm).to(dev)
        cx, cy, w, a = P[:, 0:1], P[:, 1:2], P[:, 2:3], P[:, 3:4]
        gx = torch.exp(-(x[None, :] - cx) ** 2 / (2 * w * w))
        gy = torch.exp(-(y[None, :] - cy) ** 2 / (2 * w * w))
        b = (a * gy).T @ gx
        out[k] = (b - b.mean()).reshape(-1)
    return out


def harvest_solutions(mac, sources, factor: int, rtol: float = 1e-10):
    """(inputs, targets, vcycles) for a zero-guess solve of each source on
    mac: the RMS-normalised restricted source (the residual of z0 = 0) and
    the restricted solution scaled by xxsp / rms, float32 (N, n/f, m/f), as
    harvest() pairs them."""
    torch = _torch()
    m, n = mac.m, mac.n
    H, W = n // factor, m // factor
    N = sources.shape[0]
    xs = torch.empty(N, H, W, dtype=torch.float32, device="cuda")
    ts = torch.empty(N, H, W, dtype=torch.float32, device="cuda")
    vcs = []
    for k in range(N):
        b = sources[k]
        mac.b.copy_(b)
        mac.z.zero_()
        v, _ = mac.solve_v_cycle(rtol=rtol)
        vcs.append(v)
        rms = float(torch.sqrt(torch.mean(b * b)))
        xs[k] = (_restrict(b.view(n, m), m, n, factor) / rms).float()
        ts[k] = (_restrict(mac.z.view(n, m), m, n, factor) * (mac.xxsp / rms)).float()
    return xs, ts, vcs


def evaluate_guess(net, mac, sources, factor: int, rtol: float = 1e-10):
    """Per held-out source: V-cycles to rtol from a zero guess and from the
    network's guess, the max-relative difference of the two solutions, and
    CUDA-event times of the guess and of each solve (ms)."""
    torch = _torch()
    rows = []
    for k in range(sources.shape[0]):
        mac.b.copy_(sources[k])
        mac.z.zero_()
        torch.cuda.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        e[0].record()
        v0, _ = mac.solve_v_cycle(rtol=rtol)
        e[1].record()
        z0 = mac.z.clone()
        mac.z.zero_()
        torch.cuda.synchronize()
        e[2].record()
        net.guess(mac, factor)
        e[3].record()
        e[3].synchronize()
        # the guess's error: on 8 x 8 block means (its large scales) and as
        # the starting residual relative to ||b||
        m, n = mac.m, mac.n
        err = (z0 - mac.z).view(n, m)
        blk = lambda a: a.view(n // 8, 8, m // 8, 8).mean(dim=(1, 3))
        smooth = float(torch.linalg.norm(blk(err)) / torch.linalg.norm(blk(z0.view(n, m))))
        r0 = float(torch.linalg.norm(mac.b - mac.apply()) / torch.linalg.norm(mac.b))
        e[4].record()
        v1, _ = mac.solve_v_cycle(rtol=rtol)
        e[5].record()
        e[5].synchronize()
        diff = float((mac.z - z0).abs().max() / z0.abs().max())
        rows.append(dict(v_zero=v0, v_learned=v1, rel_diff=diff, ms_zero=e[0].elapsed_time(e[1]),
                         ms_guess=e[2].elapsed_time(e[3]), ms_learned_solve=e[4].elapsed_time(e[5]),
                         smooth_err=smooth, start_resid=r0))
    return rows


def config4_experiment(m: int = 1024, n: int = 512, factor: int = 2, pairs: int = 20000, iters: int = 3000,
                       batch: int = 16, lr: float = 1e-3, heldout: int = 32, eval_grids=None, log=None):
    """Trains a U-Net on `pairs` (source, solution) pairs of the
    single-projection workload at m x n (MAC operator on square cells,
    zero-guess solves to 1e-10), seeds 0..pairs-1, and evaluates it on
    `heldout` sources of seeds 10**6 and up, on m x n and on each
    (m', n', factor') of eval_grids (the same network: m'/factor' must equal
    m/factor). Returns a summary dict."""
    import time
    from . import MgsMac
    torch = _torch()
    t0 = time.time()
    mac = MgsMac(m, n, 1. / m, 1. / m)
    xs, ts, vtrain = None, None, []
    chunk = 1000
    for c0 in range(0, pairs, chunk):
        src = gaussian_sources(m, n, range(c0, min(pairs, c0 + chunk)))
        x, t, v = harvest_solutions(mac, src, factor)
        xs = x if xs is None else torch.cat([xs, x])
        ts = t if ts is None else torch.cat([ts, t])
        vtrain += v
        del src
    t_harvest = time.time() - t0
    net = UNet(n // factor, m // factor, batch=batch, seed=7)
    t1 = time.time()
    losses = train(net, xs, ts, iters=iters, lr=lr, batch=batch, log=log)
    torch.cuda.synchronize()
    t_train = time.time() - t1
    del xs, ts
    out = {"train_grid": f"{m}x{n}", "factor": factor, "pairs": pairs, "iters": iters, "batch": batch,
           "params": net.param_count, "harvest_s": t_harvest, "train_s": t_train,
           "loss_first": float(np.mean(losses[:20])), "loss_last": float(np.mean(losses[-50:])),
           "train_vcycles_zero_guess": float(np.mean(vtrain)), "eval": {}}
    grids = [(m, n, factor)] + list(eval_grids or [])
    for (mm, nn, ff) in grids:
        mac_e = mac if (mm, nn) == (m, n) else MgsMac(mm, nn, 1. / mm, 1. / mm)
        src = gaussian_sources(mm, nn, range(10 ** 6, 10 ** 6 + heldout))
        rows = evaluate_guess(net, mac_e, src, ff)
        out["eval"][f"{mm}x{nn}"] = {
            "factor": ff, "sources": heldout,
            "vcycles_zero_guess": float(np.mean([r["v_zero"] for r in rows])),
            "vcycles_learned": float(np.mean([r["v_learned"] for r in rows])),
            "vcycles_saved": float(np.mean([r["v_zero"] - r["v_learned"] for r in rows])),
            "max_rel_diff_vs_zero_guess_solution": float(max(r["rel_diff"] for r in rows)),
            "guess_error_8x8_blocks": float(np.mean([r["smooth_err"] for r in rows])),
            "guess_start_residual": float(np.mean([r["start_resid"] for r in rows])),
            "ms_zero_guess_solve": float(np.median([r["ms_zero"] for r in rows])),
            "ms_guess": float(np.median([r["ms_guess"] for r in rows])),
            "ms_learned_solve": float(np.median([r["ms_learned_solve"] for r in rows])),
        }
        del src
    return out


if __name__ == "__main__":
    # python -m vdropimpact_b200.learned [pairs] [iters]: the learned-guess
    # experiment on the single-projection workload (training at 1024x512,
    # evaluation there and on 2048x1024 with the same network), one JSON line
    import json
    import sys
    pairs = int(sys.argv[1]) if len(sys.argv) > 1 else 20000
    iters = int(sys.argv[2]) if len(sys.argv) > 2 else 3000
    res = config4_experiment(1024, 512, 2, pairs=pairs, iters=iters, eval_grids=[(2048, 1024, 4)],
                             log=lambda it, l: print(f"iter {it} loss {l:.4g}", file=sys.stderr))
    print(json.dumps(res))
