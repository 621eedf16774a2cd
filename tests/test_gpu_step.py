"""Timestep parity on the GPU against the numpy restatement of
fluid_2d::step_forward (fluid_2d.cc:93-405), itself pinned to the
reference build. Tolerance: after every solve reaches its residual
tolerance, u, v, p and h agree within 1e-8 relative to each field's
maximum (the reference's V-cycles and the GPU's differ in smoothing order)."""
import os

import numpy as np
import pytest

from oracle import vdi_oracle as vo

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CFG = os.path.join(HERE, "golden", "id_vis32.cfg")
TOL = 1e-8
FIELDS = ("u", "v", "p", "h", "pg", "gp", "tau", "fbd")


@pytest.fixture(scope="module")
def V():
    import vdropimpact_b200 as V
    return V


def cfg_text(m=256, n=128, drop=()):
    lines = [l for l in open(CFG).read().splitlines() if l.split("#")[0].strip() not in drop
             and not l.startswith("grid_points")]
    return "\n".join(lines + [f"grid_points {m} {n}"]) + "\n"


def rel_errors(a, b):
    """Per field, max |a-b| over the field's largest |b|; and for the height
    h, which lift-off depends on near its minimum, the largest pointwise
    |a-b|/|b| as well (h_pointwise)."""
    out = {}
    for k in FIELDS:
        den = max(np.max(np.abs(b[k])), 1e-300)
        out[k] = float(np.max(np.abs(np.asarray(a[k]) - np.asarray(b[k]))) / den)
    hb = np.asarray(b["h"])
    out["h_pointwise"] = float(np.max(np.abs(np.asarray(a["h"]) - hb) / np.abs(hb)))
    return out


def test_init_fields_matches_oracle(V):
    txt = cfg_text()
    f = V.Fluid2D(txt)
    f.init_fields()
    o = vo.Oracle(vo.parse_cfg(txt))
    o.init_fields()
    e = rel_errors(f.state(), o.state())
    assert max(e.values()) == 0.0, e


@pytest.mark.parametrize("drop", [(), ("x_sym",), ("implicit_visc",)])
def test_single_step_from_oracle_state(V, drop):
    """Load the oracle's state after 5 steps, take one step on both."""
    txt = cfg_text(128, 64, drop)
    o = vo.Oracle(vo.parse_cfg(txt))
    o.init_fields()
    dt = o.prm.frame_dt()
    for _ in range(5):
        o.step(dt)
    f = V.Fluid2D(txt, mg_rtol=1e-12)
    f.load(o.state())
    o.step(dt)
    f.step_forward(dt)
    e = rel_errors(f.state(), o.state())
    assert max(e.values()) < 1e-9, e


def test_free_running_steps(V):
    """40 steps of the 256x128 workload from init, both sides free-running."""
    txt = cfg_text()
    o = vo.Oracle(vo.parse_cfg(txt))
    o.init_fields()
    dt = o.prm.frame_dt()
    f = V.Fluid2D(txt, mg_rtol=1e-10)
    f.init_fields()
    for k in range(40):
        o.step(dt)
    f.step_forward(dt, 40)
    e = rel_errors(f.state(), o.state())
    assert max(e.values()) < TOL, e
    st = f.stats()
    assert st["solves"]["MAC"] == 40 and st["solves"]["FEM"] == 40


def test_graph_replay_equals_eager(V):
    txt = cfg_text(128, 64)
    a = V.Fluid2D(txt)
    b = V.Fluid2D(txt, graph=True)
    a.init_fields(); b.init_fields()
    dt = a.frame_dt()
    a.step_forward(dt, 6)
    b.step_forward(dt, 6)
    sa, sb = a.state(), b.state()
    for k in FIELDS:
        assert np.array_equal(sa[k], sb[k]), k
    assert a.stats()["vcycles"] == b.stats()["vcycles"]


def test_mixed_precision_step(V):
    txt = cfg_text(256, 128)
    a = V.Fluid2D(txt)
    b = V.Fluid2D(txt, mg_precision="mixed")
    a.init_fields(); b.init_fields()
    dt = a.frame_dt()
    a.step_forward(dt, 10)
    b.step_forward(dt, 10)
    e = rel_errors(b.state(), a.state())
    assert max(e.values()) < TOL, e


def test_free_running_steps_odd_grid(V):
    """A 200x100 grid (a factor 25 in each side) runs every solver on the
    general multigrid hierarchy; 10 steps agree with the oracle."""
    txt = cfg_text(200, 100)
    o = vo.Oracle(vo.parse_cfg(txt))
    o.init_fields()
    dt = o.prm.frame_dt()
    f = V.Fluid2D(txt, mg_rtol=1e-10, graph=True)
    f.init_fields()
    for k in range(10):
        o.step(dt)
    f.step_forward(dt, 10)
    e = rel_errors(f.state(), o.state())
    assert max(e.values()) < TOL, e


@pytest.mark.parametrize("prec,guess", [("hybrid", "quadratic"), ("mixed", "linear")])
def test_free_running_precision_modes(V, prec, guess):
    """40 steps with FP32 coarse-grid corrections (hybrid) or FP32 V-cycles in
    FP64 refinement (mixed): every solve still stops on the FP64 residual, so
    the fields agree with the oracle within the same bound."""
    txt = cfg_text()
    o = vo.Oracle(vo.parse_cfg(txt))
    o.init_fields()
    dt = o.prm.frame_dt()
    f = V.Fluid2D(txt, mg_rtol=1e-10, mg_precision=prec, mg_guess=guess, graph=True)
    f.init_fields()
    for k in range(40):
        o.step(dt)
    f.step_forward(dt, 40)
    e = rel_errors(f.state(), o.state())
    assert max(e.values()) < TOL, e
    st = f.stats()
    assert max(st["last_rel_res"].values()) <= 1e-10


@pytest.mark.parametrize("m,n,drop", [(256, 128, ()), (200, 100, ("x_sym",)), (96, 48, ("implicit_visc",))])
def test_fused_advection_bit_identical(V, monkeypatch, m, n, drop):
    """The fused advection kernel (stages 1-5 in one launch) gives the same
    fields, bit for bit, as the four stage kernels, on grids whose sides are
    not multiples of its tile and with each boundary option."""
    txt = cfg_text(m, n, drop)
    states = {}
    for fused in ("1", "0"):
        monkeypatch.setenv("VDI_FUSED_ADVECT", fused)
        f = V.Fluid2D(txt, graph=True)
        f.init_fields()
        f.step_forward(f.frame_dt(), 20)
        states[fused] = f.state()
        f.close()
    for k in FIELDS:
        assert np.array_equal(states["1"][k], states["0"][k]), k


# ------------------------------------------- tracers and the moving frame
FRAME = os.path.join(HERE, "golden", "ref_tracers_frame_256x128.npz")


@pytest.mark.parametrize("case", ["center", "center_full"])
def test_tracers_and_frame_match_reference(V, case):
    """50 steps with tracers and the nif_center frame, with and without
    x_sym, against the reference run (ref_tracers_frame_256x128.npz):
    tracer positions and Vframe after 1 and 50 steps, fields after 50."""
    g = np.load(FRAME)
    tr = g[f"{case}_trace"]
    f = V.Fluid2D(str(g[f"{case}_cfg"]), mg_rtol=1e-12, graph=True)
    f.init_fields()
    f.set_tracers(tr[0, 2:].reshape(-1, 2))
    dt = f.frame_dt()
    span = max(f.prm.bx - f.prm.ax, f.prm.by - f.prm.ay)
    for k, steps in ((1, 1), (tr.shape[0] - 1, tr.shape[0] - 2)):
        f.step_forward(dt, steps)
        st = f.state()
        assert abs(st["Vframe"] - tr[k, 1]) <= 1e-9 * abs(tr[k, 1]), k
        assert np.max(np.abs(f.tracers().ravel() - tr[k, 2:])) <= 1e-10 * span, k
    for fld in ("u", "v", "p"):
        den = np.max(np.abs(g[f"{case}_s50_{fld}_sub"]))
        assert np.max(np.abs(st[fld][::4, ::4] - g[f"{case}_s50_{fld}_sub"])) <= TOL * den, fld
    for fld in ("h", "pg", "gp", "tau", "fbd", "ht"):
        den = max(np.max(np.abs(g[f"{case}_s50_{fld}"])), 1e-300)
        assert np.max(np.abs(st[fld] - g[f"{case}_s50_{fld}"])) <= TOL * den, fld
    assert f.stats()["kernel_launches"] > 0


@pytest.mark.parametrize("drop", [(), ("x_sym",)])
def test_nif_range_and_tracers_match_oracle(V, drop):
    """The nif_range frame (window of columns, fileinfo.cc:179-191) with 24
    tracers, 10 steps on both sides from the same tracer positions."""
    txt = cfg_text(128, 64, drop) + "tracers 24\nnif_range 4e-4\n"
    o = vo.Oracle(vo.parse_cfg(txt))
    o.init_fields()
    f = V.Fluid2D(txt, mg_rtol=1e-12)
    f.init_fields()
    f.set_tracers(o.tm.reshape(-1, 2))
    dt = o.prm.frame_dt()
    for _ in range(10):
        o.step(dt)
    f.step_forward(dt, 10)
    st = f.state()
    e = rel_errors(st, o.state())
    assert max(e.values()) < 1e-9, e
    assert st["Vframe"] == pytest.approx(o.Vframe, rel=1e-10)
    assert o.Vframe < o.prm.V
    span = max(o.prm.bx - o.prm.ax, o.prm.by - o.prm.ay)
    assert np.max(np.abs(f.tracers().ravel() - o.tm)) <= 1e-12 * span


def test_tracer_seeding_matches_reference(V, tmp_path):
    """init_fields places the tracers with the C library's rand()
    (fluid_2d.cc:495-502): in a fresh process, exactly the reference's."""
    import subprocess
    import sys
    g = np.load(FRAME)
    cfg = tmp_path / "c.cfg"
    cfg.write_text(str(g["center_cfg"]))
    out = tmp_path / "tm.npy"
    code = ("import sys, numpy as np; sys.path.insert(0, sys.argv[3]); import vdropimpact_b200 as V; "
            "f = V.Fluid2D(open(sys.argv[1]).read()); f.init_fields(); np.save(sys.argv[2], f.tracers())")
    subprocess.run([sys.executable, "-c", code, str(cfg), str(out), os.path.dirname(HERE)], check=True)
    assert np.array_equal(np.load(out).ravel(), g["center_trace"][0, 2:])

