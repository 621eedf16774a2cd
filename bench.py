"""Benchmark: Navier-Stokes timesteps per second of vdropimpact's per-step
fluid solve on the 2048x1024 liquid-deposition workload (100 cSt drop,
2048-cell gas layer), every linear solve to ||b-Az||/||b|| <= 1e-10.

One step = fluid_2d::step_forward: gas-layer Newton/tridiagonal update,
Godunov advection, MAC multigrid projection, two implicit viscous multigrid
solves, FEM multigrid projection. Solver configurations timed on the same
workload:
  plain     - FP64 V-cycles, linear time-extrapolated initial guess (the
              reference's method on the GPU)
  fast      - the headline: by default FP32 V-cycles in FP64 iterative
              refinement with the quadratic time-extrapolated guess, the
              fastest measured configuration (every solve still stops on the
              FP64 residual)
  variants  - the other configurations on the same steps: FP32 coarse-grid
              corrections (hybrid), FP64 V-cycles (fp64), FP32 V-cycles in
              FP64 refinement (mixed, when not the headline), and the learned
              U-Net guess with the refined V-cycles (learned_mixed)
`value` is the headline configuration's steps/s, summed over ranks (each
rank runs an independent replica of the simulation).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
CFG = os.path.join(ROOT, "tests", "golden", "ld_vis100.cfg")
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "vdi_ref_driver")
METRIC = "NS steps/s @2048x1024, learned+mixed MG vs plain FP64 MG, same 1e-10 residual"
WORKLOAD = "ld_vis100 drop impact, 2048x1024 liquid grid, 2048-cell gas layer"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", default="2048x1024")
    ap.add_argument("--rtol", type=float, default=1e-10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--only", default="", help="run only 'plain' or 'fast' (profiling)")
    ap.add_argument("--eager", action="store_true", help="launch kernels without CUDA graphs (profiling)")
    ap.add_argument("--fast-precision", default="mixed", choices=["fp64", "mixed", "hybrid"],
                    help="the headline configuration's V-cycles (mixed: FP32 V-cycles in FP64 refinement, "
                         "the fastest measured)")
    ap.add_argument("--fast-guess", default="quadratic", choices=["linear", "quadratic", "learned"])
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch shapes instead of the autotuned ones")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the other solver configurations (hybrid, mixed, learned+mixed)")
    return ap.parse_args()


def cfg_text(grid: str) -> str:
    m, n = grid.split("x")
    lines = [l for l in open(CFG).read().splitlines() if not l.startswith("grid_points")]
    return "\n".join(lines + [f"grid_points {m} {n}"]) + "\n"


# ------------------------------------------------------------------ dist
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def dist_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons while the
    timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------- reference
def cpu_reference(text: str, steps: int, warmup: int, threads: int | None = None) -> dict:
    """The reference's OpenMP CPU path (built from its sources by
    oracle/Makefile) timed on this host's cores."""
    import tempfile
    if not os.path.exists(REF_DRIVER):
        return {"unavailable": "oracle/_ref/vdi_ref_driver not built (make -C oracle)"}
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "bench.cfg")
        open(path, "w").write(text)
        env = dict(os.environ)
        nthreads = threads or os.cpu_count()
        env["OMP_NUM_THREADS"] = str(nthreads)
        env["VDI_MG_RTOL"] = "1e-10"
        r = subprocess.run([REF_DRIVER, "time", path, str(steps), str(warmup)], capture_output=True, text=True,
                           env=env, timeout=1800)
        if r.returncode != 0:
            return {"unavailable": f"reference driver failed: {r.stderr.strip()[:200]}"}
        out = json.loads(r.stdout.strip().splitlines()[-1])
        out["cores"] = nthreads
        return out


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return
    text = cfg_text(args.grid)
    # each "step" of this arm is one reference timestep; the run times
    # args.steps of them after args.warmup untimed ones, the same window as
    # the GPU arm (about 0.15 s per step on 16 host cores at 2048x1024)
    steps = max(1, args.steps)
    warm = max(0, args.warmup)
    r = cpu_reference(text, steps, warm)
    if "unavailable" in r:
        print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}))
        return
    v = r["steps_per_s"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": ws,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": args.grid, "solver": "reference OpenMP path + TGMG-API CPU multigrid",
                   "mg_rtol": 1e-10},
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": r["cores"], "kind": "reference",
                         "sample": f"{steps} timesteps after {warm} warm-up steps at {args.grid}"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "vcycles_per_solve": r["vcycles"] / max(r["solves"], 1),
    }
    print(json.dumps(line))


# ----------------------------------------------------------------- ours
def time_config(V, torch, text, args, precision, guess, stream, ws, clocks=None, net=None, steps=None):
    f = V.Fluid2D(text, mg_rtol=args.rtol, mg_precision=precision, mg_guess=guess, graph=not args.eager,
                  stream=stream)
    if net is not None:
        f.attach_unet(net[0], net[1])
    if not args.no_tune:
        f.autotune()
    f.init_fields()
    nsteps = steps or args.steps
    dt = f.frame_dt()
    f.step_forward(dt, args.warmup)
    f.stats(reset=True)
    barrier(ws)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if clocks:
        clocks.start()
    e0.record(stream)
    f.step_forward(dt, nsteps)
    e1.record(stream)
    e1.synchronize()
    ck = clocks.stop() if clocks else None
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ms = dist_max(ms, ws)
    st = f.stats()
    solves = sum(st["solves"].values())
    vc = {k: st["vcycles"][k] / max(st["solves"][k], 1) for k in st["vcycles"]}
    return f, dt, ms, vc, st, ck, solves


def train_guess_net(V, torch, text, args, factor=4):
    """A U-Net for the learned MAC guess, trained on the GPU on (residual,
    error) pairs harvested from the first steps of the same workload."""
    from vdropimpact_b200 import learned
    base = V.Fluid2D(text, mg_rtol=args.rtol, mg_guess="quadratic")
    base.init_fields()
    dt = base.frame_dt()
    mac = V.MgsMac(base.m, base.n, base.dx, base.dy)
    xs, ts = learned.harvest(base, 48, dt, factor, mac)
    net = learned.UNet(base.n // factor, base.m // factor, batch=8, seed=11)
    learned.train(net, xs, ts, iters=400, lr=3e-4, batch=8)
    base.close()
    return net, factor


def measured_peak_gbs():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# DRAM bytes (read + write) of one launch of the roofline kernel, from an ncu
# capture of the same kernel on a 4096x2048 grid (192.3 MB per launch),
# scaled to the 2048x1024 bench grid by the number of cells.
CC_POST_DRAM_BYTES = 192.3e6 / 4
# The same for the FP32 post-smoothing tile of the refinement's V-cycles,
# captured inside the bench's own 2048x1024 step (reads 18.9 MB: z, b and the
# coarse correction; its 8 MB of writes stay in the L2 within the launch).
CC_POST32_DRAM_BYTES = 18.92e6


def roofline(V, torch, args):
    """The dominant kernel of the step, timed with CUDA events on its own
    stream over repeated launches at the bench grid: the finest-level
    post-smoothing tile kernel of the cell-centred solves (MAC and both
    viscous systems), in the headline's V-cycle precision. Algorithmic
    bytes per launch: z in, b in, z out plus the coarse correction, 8 bytes
    a value in FP64 V-cycles, 4 in the FP32 V-cycles of the refinement."""
    m, n = (int(x) for x in args.grid.split("x"))
    s = V.MgsMac(m, n, 1.0 / m, 1.0 / m)
    g = torch.Generator(device="cuda").manual_seed(0)
    s.b.copy_(torch.randn(m * n, dtype=torch.float64, device="cuda", generator=g))
    f32 = args.fast_precision == "mixed"
    ms, nbytes = s.profile(5 if f32 else 1, 100)
    peak, kind = measured_peak_gbs()
    achieved = nbytes / (ms * 1e-3) / 1e9
    name = "cc_tile<float, POST> (FP32 V-cycle of the refinement)" if f32 else "cc_tile<double, POST>"
    out = {"kernel": f"{name} on the {args.grid} MAC grid", "bound": "hbm", "achieved": achieved,
           "peak": peak, "peak_source": kind, "unit": "GB/s", "frac": achieved / peak,
           "traffic": CC_POST32_DRAM_BYTES if f32 else CC_POST_DRAM_BYTES, "algorithmic_bytes": nbytes,
           "ms_per_launch": ms}
    if f32:
        # the FP64 tile of the FP64 configurations, for comparison
        ms64, nb64 = s.profile(1, 100)
        a64 = nb64 / (ms64 * 1e-3) / 1e9
        out["fp64_tile"] = {"kernel": f"cc_tile<double, POST> on the {args.grid} MAC grid", "achieved": a64,
                            "frac": a64 / peak, "traffic": CC_POST_DRAM_BYTES, "algorithmic_bytes": nb64,
                            "ms_per_launch": ms64}
    return out


# Canonical algorithmic bytes of the step's work outside the multigrid
# V-cycles, per liquid cell, 8-byte words: advection to the MAC source 10,
# MAC correction and advective update 11, two viscous sources 4, FEM source
# 3, velocity/pressure update 6 (34 words); and per point of each solve the
# time-extrapolated initial guess (4 words).
STEP_WORDS_PER_CELL = 34
GUESS_WORDS_PER_POINT = 4


def canonical_step(f, res, peak):
    """Step-level roofline with canonical bytes: the non-multigrid work, the
    guesses, and every V-cycle taken in the timed window at its hierarchy's
    canonical bytes per iteration."""
    st = res["stats"]
    steps = max(st["steps"], 1)
    per_iter = res["vcycle_bytes"]
    cells = f.m * f.n
    pts = {"MAC": cells, "FEM": (f.m + 1) * (f.n + 1), "VX": cells, "VY": cells}
    mg = sum(st["vcycles"][k] * per_iter[k] for k in per_iter) / steps
    guess = sum(st["solves"][k] * pts[k] for k in pts) * GUESS_WORDS_PER_POINT * 8 / steps
    other = STEP_WORDS_PER_CELL * 8 * cells
    total = mg + guess + other
    achieved = total / (res["ms"] / res["steps"] * 1e-3) / 1e9
    return {"bytes_per_step": total, "multigrid_bytes_per_step": mg, "achieved": achieved, "unit": "GB/s",
            "frac": achieved / peak}


def vcycle_rooflines(V, torch, args, sim, peak):
    """Whole FP64 V-cycles of the MAC and FEM systems of the bench grid, back
    to back as mg_test.cc:36-43 times them, against their canonical bytes."""
    m, n = (int(x) for x in args.grid.split("x"))
    out = {}
    g = torch.Generator(device="cuda").manual_seed(1)
    for name, cls, mm, nn, c1, c2 in (("MAC", V.MgsMac, m, n, sim.dx, sim.dy),
                                      ("FEM", V.MgsFem, m + 1, n + 1, sim.dx, sim.dy)):
        s = cls(mm, nn, c1, c2)
        s.b.copy_(torch.randn(mm * nn, dtype=torch.float64, device="cuda", generator=g))
        ms, nbytes = s.profile(2, 50)
        a = nbytes / (ms * 1e-3) / 1e9
        out[name] = {"ms_per_vcycle": ms, "canonical_bytes": nbytes, "achieved": a, "frac": a / peak}
        del s
    return out


def single_projection(V, torch, args, stream, peak):
    """The single-projection workload: the MAC system on a 2048x1024 grid of
    square cells (mgs_mac's operator), source the seeded zero-mean sum of 64
    Gaussians, solved from zero to 1e-10 in each precision. Reports V-cycles,
    CUDA-event time per solve and per V-cycle, canonical GB/s, and the
    max-relative difference from an FP64 solve run on past its tolerance
    (8 more V-cycles, where the iterates stop changing)."""
    m, n = 2048, 1024
    dx = 1. / m
    b = torch.from_numpy(V.projection_source(m, n, seed=2048)).cuda()
    s = V.MgsMac(m, n, dx, dx, stream=stream)
    s.b.copy_(b)
    s.z.zero_()
    s.solve_v_cycle(rtol=1e-10, precision="fp64")
    for _ in range(8):
        s.v_cycle()
    zt = s.z.clone()
    ms64, by64 = s.profile(2, 20)
    out = {"grid": f"{m}x{n}", "source": "zero-mean sum of 64 Gaussians, seed 2048", "rtol": 1e-10,
           "ms_per_fp64_vcycle_mg_test": ms64}
    cells = m * n
    for prec in ("fp64", "mixed", "hybrid"):
        for rep in range(2):     # the first solve of a precision builds its arrays
            s.z.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            v, rel = s.solve_v_cycle(rtol=1e-10, precision=prec)
            e1.record(stream)
            e1.synchronize()
        ms = e0.elapsed_time(e1)
        pts = by64 / (8 * (3. * 4 + 4.5))
        if prec == "fp64":
            per = by64
        elif prec == "hybrid":
            per = by64 / 2 + cells * (3. * 4 + 4.5) * 4
        else:
            per = by64 / 2 + 40. * cells
        err = float((s.z - zt).abs().max() / zt.abs().max())
        achieved = v * per / (ms * 1e-3) / 1e9
        out[prec] = {"vcycles": v, "rel_res": rel, "ms_per_solve": ms, "ms_per_vcycle": ms / v,
                     "canonical_bytes_per_vcycle": per, "achieved_gbs": achieved, "frac": achieved / peak,
                     "max_rel_diff_vs_fp64_converged": err}
    out["levels_points"] = pts
    return out


def e2e_run(V, torch, text, args, stream, steps, ws):
    """The same metric through the public API over the same step window as
    the timed region (a fresh simulation of the headline configuration, W
    warm-up steps from init, then the timed steps): each step is one
    Fluid2D.step_forward call (C-ABI vdi_sim_step_forward with the host
    timestep, which returns the step's device-side status), followed by a
    device-to-host read of the step's result, the gas-layer height h(x) and
    gas pressure, into pinned memory."""
    f = V.Fluid2D(text, mg_rtol=args.rtol, mg_precision=args.fast_precision, mg_guess=args.fast_guess,
                  graph=not args.eager, stream=stream)
    if not args.no_tune:
        f.autotune()
    f.init_fields()
    dt = f.frame_dt()
    f.step_forward(dt, args.warmup)
    dh, nh = f.device_field(3)
    dp, npg = f.device_field(4)
    hbuf = torch.empty(nh, dtype=torch.float64, pin_memory=True)
    pbuf = torch.empty(npg, dtype=torch.float64, pin_memory=True)
    hdev, pdev = _wrap(torch, dh, nh), _wrap(torch, dp, npg)
    barrier(ws)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        f.step_forward(dt, 1)
        with torch.cuda.stream(stream):
            hbuf.copy_(hdev, non_blocking=True)
            pbuf.copy_(pdev, non_blocking=True)
        stream.synchronize()
    e1.record(stream)
    e1.synchronize()
    ms = dist_max(e0.elapsed_time(e1), ws)
    f.close()
    return ms, 8, 8 * (nh + npg)


def _wrap(torch, ptr, n):
    """A float64 CUDA tensor viewing n doubles at device address ptr."""
    class _Iface:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                             "version": 3, "strides": None}
    return torch.as_tensor(_Iface(), device="cuda")


def main():
    args = parse()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    torch.cuda.set_device(local)
    sys.path.insert(0, ROOT)
    import vdropimpact_b200 as V
    text = cfg_text(args.grid)
    stream = torch.cuda.Stream()
    results = {}
    modes = [("plain", "fp64", "linear"), ("fast", args.fast_precision, args.fast_guess)]
    if args.only:
        modes = [m for m in modes if m[0] == args.only]
    keep = None
    for name, prec, guess in modes:
        clocks = ClockSampler(local) if name == "fast" or args.only else None
        f, dt, ms, vc, st, ck, solves = time_config(V, torch, text, args, prec, guess, stream, ws, clocks)
        results[name] = dict(ms=ms, vc=vc, clocks=ck, solves=solves, newton=st["newton_steps"],
                             launches=st["kernel_launches"], stats=st, steps=args.steps,
                             vcycle_bytes=f.vcycle_bytes())
        if name == modes[-1][0]:
            keep = (f, dt)
        else:
            f.close()
    head = results[modes[-1][0]]
    ms_step = head["ms"] / args.steps
    value = ws * 1e3 / ms_step
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.fast_precision == "fp64" else "f64+f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": args.grid, "mg_rtol": args.rtol,
                   "solver": f"{args.fast_precision} V-cycles, {args.fast_guess} time-extrapolated guess, "
                             "CUDA-graph step" + ("" if args.no_tune else ", autotuned launch shapes"),
                   "l2": "per-step working set (~0.9 GB) exceeds the 126 MB L2",
                   "parallelism": f"replicas x{ws}"},
        "clocks": head["clocks"],
        "vcycles_per_solve": head["vc"],
        "gpu_launches": head["launches"],
    }
    if "plain" in results:
        p = results["plain"]
        line["plain_fp64"] = {"steps_per_s": ws * 1e3 * args.steps / p["ms"], "ms_per_step": p["ms"] / args.steps,
                              "vcycles_per_solve": p["vc"]}
        line["speedup_vs_plain_fp64"] = p["ms"] / head["ms"]
    if not args.no_variants and not args.only and ws == 1:
        # the other solver configurations of the metric, on the same workload:
        # FP32 coarse-grid corrections, FP32 V-cycles in FP64 refinement, FP64
        # V-cycles, and the learned guess with the refined V-cycles
        vsteps = args.steps
        variants = {}
        others = [("hybrid_quadratic", "hybrid", "quadratic"), ("mixed_quadratic", "mixed", "quadratic"),
                  ("fp64_quadratic", "fp64", "quadratic"), ("learned_mixed", "mixed", "learned")]
        # the headline's own configuration is not timed twice
        others = [o for o in others if (o[1], o[2]) != (args.fast_precision, args.fast_guess)]
        for name, prec, guess in others:
            net = train_guess_net(V, torch, text, args) if guess == "learned" else None
            fv, _, msv, vcv, _, _, _ = time_config(V, torch, text, args, prec, guess, stream, ws, net=net,
                                                  steps=vsteps)
            variants[name] = {"steps_per_s": 1e3 * vsteps / msv, "steps": vsteps, "vcycles_per_solve": vcv}
            fv.close()
        line["variants"] = variants
    f, dt = keep
    line["roofline"] = roofline(V, torch, args)
    peak = line["roofline"]["peak"]
    line["roofline"]["canonical"] = {
        "note": "SURVEY-style canonical bytes (fusion-independent word counts per point) over CUDA-event time",
        "step": canonical_step(f, head, peak),
        "vcycle": vcycle_rooflines(V, torch, args, f, peak)}
    if "plain" in results:
        line["roofline"]["canonical"]["step_plain_fp64"] = canonical_step(f, results["plain"], peak)
    if not args.only and ws == 1:
        line["single_projection"] = single_projection(V, torch, args, stream, peak)
    if not args.no_e2e:
        e2e_steps = args.steps
        ms, bi, bo = e2e_run(V, torch, text, args, stream, e2e_steps, ws)
        line["e2e"] = {"value": ws * 1e3 * e2e_steps / ms, "unit": "steps/s", "h2d_bytes_per_step": bi,
                       "d2h_bytes_per_step": bo}
    f.close()
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        r = cpu_reference(text, 8, 2)
        if "unavailable" not in r:
            line["cpu_baseline"] = {"value": r["steps_per_s"], "unit": "steps/s", "cores": r["cores"],
                                    "kind": "reference",
                                    "sample": f"8 timesteps of the same workload after 2 warm-up steps"}
        else:
            line["cpu_baseline"] = {"value": None, "unavailable": r["unavailable"]}
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
