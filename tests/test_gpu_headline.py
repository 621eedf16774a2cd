"""Parity at the sizes the measurements use, against the reference build
itself (oracle/_ref/vdi_ref_driver: the reference's unmodified sources on a
CPU multigrid that stops at ||b-Az||/||b|| <= 1e-10).

- The liquid-deposition case (sims/ld_vis100.cfg physics) on its 2048x1024
  grid with a 2048-cell gas layer: 100 steps of fluid_2d::step_forward
  (fluid_2d.cc:93-405) from init_fields, with the solver configurations
  that are timed (FP64 V-cycles, and FP32 V-cycles in FP64 refinement; the
  quadratic time-extrapolated guess, autotuned launch shapes and hierarchy
  cuts, CUDA-graph steps, the separable exact coarse solve).
- Members of a batched viscosity sweep at 512x256 and 1024x512 (the sweep of
  sims/create_cfg.pl:11), stepped together in one batch with FP32 V-cycles
  in FP64 refinement, each against its own reference run.

Tolerance: after every solve reaches 1e-10, u, v, p, pg, gp and fbd agree
within 1e-8 of each field's largest magnitude, and the gas-layer height h
within 1e-8 of its own value at every point, the minimum (where lift-off is
decided) included. The shear stress tau = -(mu_g/2) h dp/dx
(gas_layer_solve.cc:248) carries the height as a factor, which grows as x^2
towards the far field, so a difference of the pressure gradient there that
is 1e-10 of its own scale becomes 1e-6 of tau's largest value near the axis;
tau is therefore compared through its pressure-gradient factor tau/h. That
factor is a derivative: differencing a pressure that agrees to a few 1e-11
of its scale across features hundreds of cells wide leaves it at about 2e-8
of its own scale, so it is held to 1e-7 (and tau's two never-written ghost
entries, quirk Q1, exactly)."""
import os
import subprocess

import numpy as np
import pytest

from oracle import vdi_oracle as vo

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-8
TOL_TAU_OVER_H = 1e-7
SCALED = ("u", "v", "p", "pg", "gp", "fbd")


@pytest.fixture(scope="module")
def V():
    import vdropimpact_b200 as V
    return V


def cfg_text(name, m, n):
    lines = [l for l in open(os.path.join(HERE, "golden", name)).read().splitlines()
             if not l.startswith("grid_points")]
    return "\n".join(lines + [f"grid_points {m} {n}"]) + "\n"


def reference_state(ref_driver, tmp_path, tag, text, nsteps):
    cfg = tmp_path / f"{tag}.cfg"
    cfg.write_text(text)
    out = tmp_path / f"{tag}.bin"
    env = dict(os.environ, VDI_MG_RTOL="1e-10", OMP_NUM_THREADS=str(os.cpu_count()))
    subprocess.run([ref_driver, "step", str(cfg), str(nsteps), str(out)], check=True, capture_output=True,
                   env=env, timeout=1200)
    return vo.read_states(str(out))[0]


def field_errors(a, b):
    """Per field: max |a-b| over the field's largest |b|; for h the largest
    pointwise |a-b|/|b|, and the same at the point of b's minimum."""
    out = {}
    for k in SCALED:
        den = max(np.max(np.abs(b[k])), 1e-300)
        out[k] = float(np.max(np.abs(np.asarray(a[k]) - np.asarray(b[k]))) / den)
    h, hr = np.asarray(a["h"]), np.asarray(b["h"])
    assert np.all(hr > 0)
    m = hr.size
    ta, tr = np.asarray(a["tau"]), np.asarray(b["tau"])
    ga, gr = ta[:m] / hr, tr[:m] / hr
    out["tau_over_h"] = float(np.max(np.abs(ga - gr)) / max(np.max(np.abs(gr)), 1e-300))
    assert np.array_equal(ta[m:m + 2], tr[m:m + 2])
    out["h_pointwise"] = float(np.max(np.abs(h - hr) / hr))
    i = int(np.argmin(hr))
    out["h_at_min"] = float(abs(h[i] - hr[i]) / hr[i])
    return out


LD_STEPS = 100


@pytest.fixture(scope="module")
def ld_reference(ref_driver, tmp_path_factory):
    """The reference's 100 steps of the 2048x1024 case, run once."""
    text = cfg_text("ld_vis100.cfg", 2048, 1024)
    return reference_state(ref_driver, tmp_path_factory.mktemp("ld"), "ld", text, LD_STEPS)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_liquid_deposition_2048x1024_matches_reference(V, ld_reference, precision):
    text = cfg_text("ld_vis100.cfg", 2048, 1024)
    nsteps = LD_STEPS
    f = V.Fluid2D(text, mg_rtol=1e-10, mg_precision=precision, mg_guess="quadratic", graph=True)
    f.autotune()
    f.init_fields()
    dt = f.frame_dt()
    f.step_forward(dt, nsteps)
    a = f.state()
    st = f.stats()
    f.close()
    r = ld_reference
    assert a["time"] == pytest.approx(r["time"], rel=1e-14)
    e = field_errors(a, r)
    print(f"2048x1024 ld_vis100, 100 steps, {precision}:", e, "V-cycles", st["vcycles"])
    assert e.pop("tau_over_h") < TOL_TAU_OVER_H
    assert max(e.values()) < TOL, e
    assert st["solves"]["MAC"] == nsteps and st["solves"]["FEM"] == nsteps


def _sweep_members(V, sizes, seed):
    """The first member of a seeded sweep at each requested grid width."""
    cfgs = V.sweep_configs(64, seed=seed, sizes=(256, 512, 1024))
    out = []
    for m in sizes:
        out.append(next(c for c in cfgs if f"grid_points {m} {m // 2}" in c))
    return out


def test_batch_members_512_and_1024_match_reference(V, ref_driver, tmp_path):
    cfgs = _sweep_members(V, (512, 1024), seed=0)
    nsteps = 10
    b = V.Batch(cfgs, mg_rtol=1e-10, mg_precision="mixed", mg_guess="quadratic")
    b.autotune()
    b.init_fields()
    dts = b.frame_dts()
    b.step_forward(dts, nsteps)
    states = [s.state() for s in b.sims]
    b.close()
    for k, text in enumerate(cfgs):
        r = reference_state(ref_driver, tmp_path, f"b{k}", text, nsteps)
        assert states[k]["time"] == pytest.approx(r["time"], rel=1e-14)
        e = field_errors(states[k], r)
        print(f"batch member {k} ({states[k]['m']}x{states[k]['n']}):", e)
        assert e.pop("tau_over_h") < TOL_TAU_OVER_H, k
        assert max(e.values()) < TOL, (k, e)
