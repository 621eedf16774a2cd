"""B200 implementation of vdropimpact's per-timestep fluid solve.

Python host-side mirror of the reference's classes, over the C ABI of
include/vdi.h (libvdi.so):

    Fluid2D      fluid_2d      (fluid_2d.hh:21-142): init_fields,
                 step_forward, timestep_select, solve, restart-style state
    MgsMac       mgs_mac       (mgs_mac.hh:25-75)  : solve_v_cycle, v_cycle
    MgsFem       mgs_fem       (mgs_fem.hh:36-82)  : solve_v_cycle, v_cycle
    ViscoImpl    visco_impl    (visco_impl.hh:17-58): setup_and_solve
    TriSolve     tri_solve     (tri_solve.hh:6-22) : solve_lapack

Errors the reference reports with fatal_error()/exit() raise VdiError.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import (VDI_MG_FP64, VDI_MG_MIXED, VDI_GUESS_EXTRAPOLATE, VDI_GUESS_LEARNED, VDI_MG_MAC,
                   VDI_MG_FEM, VDI_MG_VISC_U, VDI_MG_VISC_V, VdiError, check, lib)

__all__ = ["Fluid2D", "MgsMac", "MgsMacNeumann", "MgsFem", "ViscoImpl", "TriSolve", "VdiError", "params_from_cfg",
           "VDI_MG_FP64", "VDI_MG_MIXED", "VDI_GUESS_EXTRAPOLATE", "VDI_GUESS_LEARNED", "projection_source"]

_PREC = {"fp64": VDI_MG_FP64, "mixed": VDI_MG_MIXED, "hybrid": _abi.VDI_MG_HYBRID, VDI_MG_FP64: VDI_MG_FP64,
         VDI_MG_MIXED: VDI_MG_MIXED, _abi.VDI_MG_HYBRID: _abi.VDI_MG_HYBRID}


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("vdropimpact_b200 needs a CUDA device")
    return torch


def _stream_handle(stream):
    if stream is None:
        return None
    return C.c_void_p(int(getattr(stream, "cuda_stream", stream)))


def params_from_cfg(cfg: str) -> _abi.VdiParams:
    """fileinfo::fileinfo (fileinfo.cc:11-193) for a path ending in .cfg or
    for configuration text."""
    text = open(cfg).read() if (cfg.endswith(".cfg") and os.path.exists(cfg)) else cfg
    p = _abi.VdiParams()
    check(lib().vdi_params_from_cfg(text.encode(), C.byref(p)), "vdi_params_from_cfg")
    return p


class Fluid2D:
    """fluid_2d (fluid_2d.hh:21-142) on the GPU."""

    GUESS = {"linear": 0, "learned": 1, "quadratic": 2}

    def __init__(self, cfg, *, mg_rtol: float = 1e-10, mg_max_vcycles: int = 200,
                 mg_precision="fp64", mg_guess="linear", graph: bool = False, stream=None):
        self.prm = cfg if isinstance(cfg, _abi.VdiParams) else params_from_cfg(cfg)
        self.prm.mg_rtol = mg_rtol
        self.prm.mg_guess = self.GUESS[mg_guess] if isinstance(mg_guess, str) else int(mg_guess)
        self.prm.mg_max_vcycles = mg_max_vcycles
        self.prm.mg_precision = _PREC[mg_precision]
        self.m, self.n = self.prm.m, self.prm.n
        self.me, self.ne, self.ml = self.m + 1, self.n + 1, self.m + 4
        self.dx = (self.prm.bx - self.prm.ax) / self.m
        self.dy = (self.prm.by - self.prm.ay) / self.n
        h = C.c_void_p()
        check(lib().vdi_sim_create(C.byref(self.prm), _stream_handle(stream), C.byref(h)), "vdi_sim_create")
        self._h = h
        if graph:
            self.use_graph(True)

    # ------------------------------------------------------------------
    @classmethod
    def _view(cls, handle, prm, owner):
        """A simulation owned by a Batch (not destroyed by this object)."""
        f = cls.__new__(cls)
        f.prm = prm
        f.m, f.n = prm.m, prm.n
        f.me, f.ne, f.ml = f.m + 1, f.n + 1, f.m + 4
        f.dx = (prm.bx - prm.ax) / f.m
        f.dy = (prm.by - prm.ay) / f.n
        f._h = handle
        f._owner = owner
        return f

    def close(self):
        if getattr(self, "_owner", None) is not None:
            self._h = None
            return
        if getattr(self, "_h", None):
            lib().vdi_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------
    def init_fields(self):
        """fluid_2d::init_fields (fluid_2d_sio.cc:14-35)."""
        check(lib().vdi_sim_init_fields(self._h), "vdi_sim_init_fields")

    def timestep_select(self, interval: float):
        """fluid_2d::timestep_select (fluid_2d.hh:82-86): returns (l, adt)."""
        adt = C.c_double()
        l = C.c_int()
        check(lib().vdi_sim_timestep_select(self._h, interval, C.byref(adt), C.byref(l)), "timestep_select")
        return l.value, adt.value

    def frame_dt(self) -> float:
        """The timestep of fluid_2d::solve (fluid_2d.cc:42)."""
        return self.timestep_select(self.prm.t_end / self.prm.nframes)[1]

    def step_forward(self, dt: float, nsteps: int = 1):
        """fluid_2d::step_forward (fluid_2d.cc:93-405), nsteps times."""
        check(lib().vdi_sim_step_forward(self._h, dt, nsteps), "vdi_sim_step_forward")

    def use_graph(self, enable: bool = True):
        check(lib().vdi_sim_use_graph(self._h, int(enable)), "vdi_sim_use_graph")

    def synchronize(self):
        check(lib().vdi_sim_synchronize(self._h), "vdi_sim_synchronize")

    def solve(self, frames: int | None = None, callback=None):
        """fluid_2d::solve (fluid_2d.cc:40-89) without file output: steps
        `frames` frames of l steps each and calls callback(k, self)."""
        l, adt = self.timestep_select(self.prm.t_end / self.prm.nframes)
        for k in range(1, (frames or self.prm.nframes) + 1):
            self.step_forward(adt, l)
            if callback:
                callback(k, self)

    # ------------------------------------------------------------------
    def _arrays(self):
        m, n = self.m, self.n
        ng = (m + 4) * (n + 4)
        return dict(u=np.zeros(ng), v=np.zeros(ng), p=np.zeros(ng), gp=np.zeros(m + 1),
                    tau=np.zeros(m + 4), h=np.zeros(m), fbd=np.zeros(m), pg=np.zeros(m + 1), ht=np.zeros(m))

    @staticmethod
    def _ptr(a):
        return a.ctypes.data_as(_abi._dp)

    def state(self) -> dict:
        """The restart-file state (fluid_2d_sio.cc:97-119,
        gas_layer_solve.cc:323-329) as numpy arrays; u, v, p have shape
        (n+4, m+4)."""
        a = self._arrays()
        st = _abi.VdiState()
        for k, v in a.items():
            setattr(st, k, self._ptr(v))
        check(lib().vdi_sim_get_state(self._h, C.byref(st)), "vdi_sim_get_state")
        shp = (self.n + 4, self.m + 4)
        out = dict(m=self.m, n=self.n, time=st.time, Vframe=st.Vframe)
        for k, v in a.items():
            out[k] = v.reshape(shp) if k in ("u", "v", "p") else v
        return out

    def load(self, s: dict):
        """Loads a state (the restart loader, fluid_2d_sio.cc:39-62); the
        multigrid time-extrapolation history restarts as in the reference."""
        keep = {}
        st = _abi.VdiState()
        st.time = float(s["time"])
        st.Vframe = float(s["Vframe"])
        for k in ("u", "v", "p", "gp", "tau", "h", "fbd", "pg", "ht"):
            a = np.ascontiguousarray(s[k], dtype=np.float64).ravel()
            keep[k] = a
            setattr(st, k, self._ptr(a))
        check(lib().vdi_sim_set_state(self._h, C.byref(st)), "vdi_sim_set_state")

    def tracers(self) -> np.ndarray:
        """Tracer positions, shape (ntrace, 2): the reference's tm array
        (fluid_2d.hh:49-50), moved each step by fluid_2d::update_tracers."""
        out = np.zeros(2 * self.prm.ntrace)
        check(lib().vdi_sim_get_tracers(self._h, self._ptr(out), out.size), "vdi_sim_get_tracers")
        return out.reshape(-1, 2)

    def set_tracers(self, xy):
        """Places the tracers (ntrace x 2 positions)."""
        a = np.ascontiguousarray(xy, dtype=np.float64).ravel()
        check(lib().vdi_sim_set_tracers(self._h, self._ptr(a), a.size), "vdi_sim_set_tracers")

    def stats(self, reset: bool = False) -> dict:
        s = _abi.VdiStats()
        check(lib().vdi_sim_stats(self._h, C.byref(s), int(reset)), "vdi_sim_stats")
        names = ("MAC", "FEM", "VX", "VY")
        return dict(steps=s.steps, solves=dict(zip(names, list(s.solves))),
                    vcycles=dict(zip(names, list(s.vcycles))), newton_steps=s.newton_steps,
                    tri_pivot_fallbacks=s.tri_pivot_fallbacks,
                    height_fixed_point_iters=s.height_fixed_point_iters,
                    last_rel_res=dict(zip(names, list(s.last_rel_res))), kernel_launches=s.kernel_launches)

    def autotune(self) -> dict:
        """Times the candidate launch shapes of the stencil kernels and the
        tile/CTA cut of each multigrid hierarchy on this grid, and keeps the
        fastest (cached per grid in the process)."""
        t = _abi.VdiTune()
        check(lib().vdi_sim_autotune(self._h, C.byref(t)), "vdi_sim_autotune")
        return _tune_dict(t)

    PROFILE = {"advect": 0, "advect_stages": 1, "gas": 2, "liftoff": 3}

    def profile(self, part: str, iters: int = 20) -> float:
        """Mean ms per launch of one part of the step (measurement only: it
        overwrites intermediate arrays and, for "gas" and "liftoff", advances
        the gas layer or the lift-off search)."""
        ms = C.c_float()
        check(lib().vdi_sim_profile(self._h, self.PROFILE[part], iters, C.byref(ms)), "vdi_sim_profile")
        return ms.value

    LIFTOFF = {"off": 0, "smoothed": 1, "raw": 2}

    def liftoff_setup(self, mode="smoothed", every: int = 1, history: int = 0):
        """Configures the device lift-off search (tt_analysis.cc:97-171):
        mode "smoothed" (the tool's default), "raw" (its -r flag) or "off";
        a state every `every` steps; `history` per-state minima kept."""
        check(lib().vdi_sim_liftoff_setup(self._h, self.LIFTOFF[mode], every, history), "vdi_sim_liftoff_setup")
        self._lhist = history

    def liftoff(self) -> dict:
        """The search so far: the lift-off state and its minimum, the tool's
        summary times, and the per-state minima kept (xmin, hmin arrays)."""
        out = _abi.VdiLiftoff()
        cap = getattr(self, "_lhist", 0)
        xs = np.zeros(max(cap, 1))
        fs = np.zeros(max(cap, 1))
        check(lib().vdi_sim_liftoff(self._h, C.byref(out), xs.ctypes.data_as(C.c_void_p),
                                    fs.ctypes.data_as(C.c_void_p), cap), "vdi_sim_liftoff")
        n = min(cap, out.states)
        d = {k: getattr(out, k) for k, *_ in out._fields_}
        d["xmin"], d["hmin"] = xs[:n].copy(), fs[:n].copy()
        return d

    def attach_unet(self, net, factor: int):
        """Uses net (learned.UNet, trained on this grid restricted by factor)
        as the MAC solve's learned initial-guess correction."""
        check(lib().vdi_sim_attach_unet(self._h, net._h, factor, float(net.out_scale)), "vdi_sim_attach_unet")
        self._unet = net

    def vcycle_bytes(self, precision=None) -> dict:
        """Canonical algorithmic bytes of one solve-loop iteration of each
        multigrid system (measurement helper; see vdi_sim_vcycle_bytes)."""
        out = (C.c_double * 4)()
        prec = _PREC[precision if precision is not None else self.prm.mg_precision]
        check(lib().vdi_sim_vcycle_bytes(self._h, prec, out), "vdi_sim_vcycle_bytes")
        return dict(zip(("MAC", "FEM", "VX", "VY"), list(out)))

    def device_field(self, which: int):
        p = _abi._dp()
        n = C.c_size_t()
        check(lib().vdi_sim_device_field(self._h, which, C.byref(p), C.byref(n)), "vdi_sim_device_field")
        return C.cast(p, C.c_void_p).value, n.value


def _tune_dict(t) -> dict:
    return dict(block=(t.blk_x, t.blk_y), cta_limit=list(t.cta_limit), tiled_levels=list(t.tiled_levels),
                stencil_ms=t.stencil_ms, vcycle_ms=list(t.vcycle_ms), from_cache=bool(t.from_cache))


class Batch:
    """Independent simulations stepped together, one CUDA graph (a branch
    per simulation) per timestep. cfgs: .cfg texts or VdiParams."""

    def __init__(self, cfgs, *, mg_rtol: float = 1e-10, mg_max_vcycles: int = 200, mg_precision="fp64",
                 mg_guess="linear"):
        prms = []
        for c in cfgs:
            p = c if isinstance(c, _abi.VdiParams) else params_from_cfg(c)
            p.mg_rtol = mg_rtol
            p.mg_max_vcycles = mg_max_vcycles
            p.mg_precision = _PREC[mg_precision]
            p.mg_guess = Fluid2D.GUESS[mg_guess] if isinstance(mg_guess, str) else int(mg_guess)
            prms.append(p)
        arr = (_abi.VdiParams * len(prms))(*prms)
        h = C.c_void_p()
        check(lib().vdi_batch_create(arr, len(prms), C.byref(h)), "vdi_batch_create")
        self._h = h
        self.sims = []
        for k, p in enumerate(prms):
            sh = C.c_void_p()
            check(lib().vdi_batch_sim(h, k, C.byref(sh)), "vdi_batch_sim")
            self.sims.append(Fluid2D._view(sh, p, self))

    def __len__(self):
        return len(self.sims)

    def close(self):
        if getattr(self, "_h", None):
            for s in self.sims:
                s._h = None
            lib().vdi_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_fields(self):
        check(lib().vdi_batch_init_fields(self._h), "vdi_batch_init_fields")

    def frame_dts(self):
        return [s.frame_dt() for s in self.sims]

    def autotune(self):
        out = (_abi.VdiTune * len(self.sims))()
        check(lib().vdi_batch_autotune(self._h, out), "vdi_batch_autotune")
        return [_tune_dict(t) for t in out]

    def step_forward(self, dts, nsteps: int = 1):
        arr = (C.c_double * len(self.sims))(*[float(d) for d in dts])
        check(lib().vdi_batch_step_forward(self._h, arr, nsteps), "vdi_batch_step_forward")


def sweep_configs(count: int, seed: int = 0, sizes=(256, 512, 1024)):
    """A seeded viscosity / impact-velocity sweep in the manner of the
    reference's sims/create_cfg.pl: viscosity log-uniform in 1-100 cSt, impact
    velocity uniform in 0.2-0.5 m/s, grid m x m/2 with m drawn from sizes; the
    larger domain (L_nd 45, t_end_nd 100) from 25 cSt up, as create_cfg.pl
    switches it. Returns .cfg texts."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nu = float(np.exp(rng.uniform(np.log(1.0), np.log(100.0))))
        V = float(rng.uniform(0.2, 0.5))
        m = int(rng.choice(sizes))
        big = nu >= 25
        out.append("\n".join([
            f"grid_points {m} {m // 2}", f"L_nd {45 if big else 30}", "h0_nd 15",
            f"t_end_nd {100 if big else 50}", "frames 250", "tmult 8e-3", f"nul_cSt {nu:.6g}", "rhol 997.96",
            "R 1.5e-3", f"V {V:.6g}", "gamma 1.4", "sigma 72e-3", "mug 1.820775e-5", "Pamb 1e5", "x_sym",
            "implicit_visc", "gas_layer_model"]) + "\n")
    return out


def projection_source(m: int, n: int, seed: int, count: int = 64) -> np.ndarray:
    """The source of the single-projection workload on an m x n cell grid of
    a domain 1 wide and n/m high: the sum of `count` Gaussians (centres
    uniform over the domain, widths uniform in 0.01-0.1 of its width,
    amplitudes N(0,1), drawn from a generator seeded with `seed`), minus its
    mean; float64, m*n values in the row order ij = i + m*j of mgs_mac."""
    rng = np.random.default_rng(seed)
    x = (np.arange(m) + 0.5) / m
    y = (np.arange(n) + 0.5) / n * (n / m)
    b = np.zeros((n, m))
    for _ in range(count):
        cx, cy = rng.uniform(0, 1), rng.uniform(0, n / m)
        w = rng.uniform(0.01, 0.1)
        a = rng.standard_normal()
        gx = np.exp(-(x - cx) ** 2 / (2 * w * w))
        gy = np.exp(-(y - cy) ** 2 / (2 * w * w))
        b += a * np.outer(gy, gx)
    return (b - b.mean()).ravel()


def sweep_cost(cfg: str) -> float:
    """Relative cost of running one .cfg to its end: cells times timesteps
    (the frame interval over the timestep of fluid_2d.hh:82-86, times the
    frames)."""
    p = params_from_cfg(cfg)
    dx = (p.bx - p.ax) / p.m
    rho, mu = p.rho, p.mu
    dt_reg = dx * p.tmult if p.implicit_visc else dx * dx * rho / mu * p.tmult * 0.25
    steps_per_frame = int((p.t_end / p.nframes) / dt_reg) + 1
    return float(p.m) * p.n * steps_per_frame * p.nframes


def shard_sweep(cfgs, rank: int, world: int):
    """The indices of the simulations of a sweep that rank `rank` of `world`
    runs: longest first onto the least-loaded rank (ties to the lower rank),
    by sweep_cost. Every rank computes the same assignment from the same
    list, so ranks need no exchange; the simulations are independent and a
    rank runs its share as one Batch."""
    if not (0 <= rank < world):
        raise ValueError("rank must lie in [0, world)")
    costs = [sweep_cost(c) for c in cfgs]
    order = sorted(range(len(cfgs)), key=lambda k: (-costs[k], k))
    load = [0.0] * world
    mine = []
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += costs[k]
        if r == rank:
            mine.append(k)
    return sorted(mine)


def profile_min(h, ax: float, dx: float, mode: str = "smoothed"):
    """(x, height) of the minimum of one height profile (a float64 CUDA
    tensor of m cell values) as the reference's analysis tool finds it
    (tt_analysis.cc:111-146)."""
    torch = _torch()
    h = h.contiguous()
    xm, fm = C.c_double(), C.c_double()
    torch.cuda.synchronize()
    check(lib().vdi_profile_min(h.numel(), ax, dx, Fluid2D.LIFTOFF[mode], C.c_void_p(h.data_ptr()), None,
                                C.byref(xm), C.byref(fm)), "vdi_profile_min")
    return xm.value, fm.value


class _MgSystem:
    """Common part of the TGMG-style problem classes: a device solution z and
    source b (torch float64 tensors on the current CUDA device) and the
    solver calls of tgmg (mg_test.cc:20-45)."""

    kind = None
    precision = "fp64"

    def __init__(self, m, n, c1, c2, x_sym=False, stream=None):
        torch = _torch()
        self.m, self.n, self.mn = m, n, m * n
        self.z = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        self.b = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        self._stream = stream
        h = C.c_void_p()
        check(lib().vdi_mg_create(self.kind, m, n, c1, c2, int(x_sym), _stream_handle(stream), C.byref(h)),
              "vdi_mg_create")
        self._h = h
        self.last = None

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                lib().vdi_mg_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def setup(self):
        check(lib().vdi_mg_setup(self._h), "vdi_mg_setup")

    def solve_v_cycle(self, rtol: float = 1e-10, max_vcycles: int = 200, precision=None):
        """tgmg::solve_v_cycle: V-cycles on z from its current value until
        ||b-Az||/||b|| <= rtol. Returns (vcycles, relative residual)."""
        _torch().cuda.synchronize()
        r = _abi.VdiMgResult()
        check(lib().vdi_mg_solve(self._h, C.c_void_p(self.b.data_ptr()), C.c_void_p(self.z.data_ptr()),
                                 rtol, max_vcycles, _PREC[precision or self.precision], C.byref(r)),
              "vdi_mg_solve")
        self.last = (r.vcycles, r.rel_res)
        return self.last

    def v_cycle(self):
        """tgmg::v_cycle: one FP64 V-cycle on z."""
        _torch().cuda.synchronize()
        check(lib().vdi_mg_v_cycle(self._h, C.c_void_p(self.b.data_ptr()), C.c_void_p(self.z.data_ptr())),
              "vdi_mg_v_cycle")

    def apply(self, z=None):
        """A z (a_cc*z + mul_a of the problem class)."""
        torch = _torch()
        z = self.z if z is None else z
        y = torch.empty_like(z)
        torch.cuda.synchronize()
        check(lib().vdi_mg_apply(self._h, C.c_void_p(z.data_ptr()), C.c_void_p(y.data_ptr())), "vdi_mg_apply")
        return y

    def profile(self, which: int = 1, iters: int = 50):
        """Mean duration (ms) and algorithmic bytes of one launch of the
        finest-level pre- (0) or post- (1) smoothing kernel."""
        ms = C.c_float()
        by = C.c_double()
        _torch().cuda.synchronize()
        check(lib().vdi_mg_profile(self._h, which, iters, C.c_void_p(self.b.data_ptr()),
                                   C.c_void_p(self.z.data_ptr()), C.byref(ms), C.byref(by)), "vdi_mg_profile")
        return ms.value, by.value

    def coarse_cycle(self, precision=None):
        """(first level, CTAs) of the coarse path of a V-cycle in this
        precision: CTAs 1 for one CTA, 8 or 16 for a cluster, 0 for the
        dense-inverse solve over the whole GPU, -1 for the separable
        transform solve; first level -1 when the hierarchy has none."""
        first, ctas = C.c_int(), C.c_int()
        check(lib().vdi_mg_coarse_cycle(self._h, _PREC[precision or self.precision], C.byref(first),
                                        C.byref(ctas)), "vdi_mg_coarse_cycle")
        return first.value, ctas.value

    def residual(self):
        """(r, ||r||_2) with r = b - A z (tgmg::output_res)."""
        torch = _torch()
        r = torch.empty_like(self.z)
        nrm = C.c_double()
        torch.cuda.synchronize()
        check(lib().vdi_mg_residual(self._h, C.c_void_p(self.b.data_ptr()), C.c_void_p(self.z.data_ptr()),
                                    C.c_void_p(r.data_ptr()), C.byref(nrm)), "vdi_mg_residual")
        return r, nrm.value


class MgsMac(_MgSystem):
    """mgs_mac(int m,int n,double dx,double dy,double* b) (mgs_mac.cc:23-27)."""
    kind = VDI_MG_MAC

    def __init__(self, m, n, dx, dy, stream=None):
        super().__init__(m, n, dx, dy, False, stream)
        self.xxsp, self.yysp = 1. / (dx * dx), 1. / (dy * dy)


class MgsMacNeumann(_MgSystem):
    """The MAC operator with Neumann conditions on all four sides (a pure
    Neumann pressure Poisson problem, which the reference does not have): the
    solve removes the source's mean (its compatibility condition) and returns
    the zero-mean solution."""
    kind = _abi.VDI_MG_MAC_NEUMANN

    def __init__(self, m, n, dx, dy, stream=None):
        super().__init__(m, n, dx, dy, False, stream)


class MgsFem(_MgSystem):
    """mgs_fem(int m,int n,double dx,double dy,double* b) (mgs_fem.cc:26-30);
    m x n nodes."""
    kind = VDI_MG_FEM

    def __init__(self, m, n, dx, dy, stream=None):
        super().__init__(m, n, dx, dy, False, stream)


class ViscoImpl(_MgSystem):
    """visco_impl (visco_impl.hh:17-58) on an m x n grid."""

    def __init__(self, m, n, x_sym: bool, horizontal_vel: bool, vfx=1., vfy=1., stream=None):
        self.kind = VDI_MG_VISC_U if horizontal_vel else VDI_MG_VISC_V
        self.x_sym, self.horizontal_vel = x_sym, horizontal_vel
        self.vfx, self.vfy = vfx, vfy
        super().__init__(m, n, vfx, vfy, x_sym, stream)

    def setup_and_solve(self, vfx, vfy, rtol=1e-10, max_vcycles=200, precision=None):
        """visco_impl::setup_and_solve (visco_impl.cc:21-39) without the time
        extrapolation (the caller supplies z)."""
        if abs(vfx - self.vfx) > 1e2 * np.finfo(float).eps * self.vfx or vfy != self.vfy:
            h = C.c_void_p()
            check(lib().vdi_mg_create(self.kind, self.m, self.n, vfx, vfy, int(self.x_sym),
                                      _stream_handle(self._stream), C.byref(h)), "vdi_mg_create")
            lib().vdi_mg_destroy(self._h)
            self._h = h
            self.vfx, self.vfy = vfx, vfy
        return self.solve_v_cycle(rtol, max_vcycles, precision)


class TriSolve:
    """tri_solve (tri_solve.hh:6-22): host arrays a, b, c, d of length m;
    solve_lapack() solves on the GPU and leaves the solution in d."""

    def __init__(self, m: int):
        self.m = m
        self.a = np.zeros(m)
        self.b = np.zeros(m)
        self.c = np.zeros(m)
        self.d = np.zeros(m)
        self.pivoted = False

    def solve_lapack(self):
        torch = _torch()
        dev = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (self.a, self.b, self.c, self.d)]
        piv = C.c_int()
        torch.cuda.synchronize()
        check(lib().vdi_tri_solve(self.m, *[C.c_void_p(t.data_ptr()) for t in dev], None, C.byref(piv)),
              "vdi_tri_solve")
        self.d = dev[3].cpu().numpy()
        self.pivoted = bool(piv.value)
        return self.d
