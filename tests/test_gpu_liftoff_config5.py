"""The lift-off run at scale: ld_vis100 on its 2048x1024 grid for 20,000
steps, with the lift-off search of tt_analysis.cc:97-171 (smoothed heights,
every step) running on the device, in the two configurations the bench
times fastest: FP64 V-cycles and FP32 V-cycles in FP64 refinement, both with
the quadratic time-extrapolated guess and every solve to 1e-10.

The two runs must find lift-off at the same state (within one step) and
agree on the minimum gas-layer height there to 1e-7 of its value: each
solve leaves an error of about 1e-10 of its scale, and 20,000 steps of such
solves drift apart by a few 1e-8 at most (an FP64-against-FP64 comparison
of the linear and quadratic guesses over the same run differed by 2e-9).
Both must also reproduce the state and height this configuration first
gave (18462, 2.2725481e-7), the same tolerances. The reference's CPU code
would take about 50 minutes for this run, so it is compared over 100 steps
in test_gpu_headline.py instead."""
import os

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
STEPS = 20000
STATE, HMIN = 18462, 2.2725481e-7


def _run(V, precision):
    text = open(os.path.join(HERE, "golden", "ld_vis100.cfg")).read()
    f = V.Fluid2D(text, mg_rtol=1e-10, mg_precision=precision, mg_guess="quadratic", graph=True)
    f.autotune()
    f.liftoff_setup("smoothed", 1, 0)
    f.init_fields()
    dt = f.frame_dt()
    f.step_forward(dt, STEPS)
    r = f.liftoff()
    st = f.stats()
    f.close()
    return r, st


def test_liftoff_at_scale_in_both_precisions():
    import vdropimpact_b200 as V
    res = {p: _run(V, p) for p in ("fp64", "mixed")}
    for p, (r, st) in res.items():
        print(p, "lift-off state", r["min_state"], "minimum height", r["min_height"], "V-cycles", st["vcycles"])
        assert r["states"] == STEPS + 1
        assert abs(r["min_state"] - STATE) <= 1, (p, r["min_state"])
        assert abs(r["min_height"] - HMIN) <= 1e-7 * HMIN, (p, r["min_height"])
    a, b = res["fp64"][0], res["mixed"][0]
    assert abs(a["min_state"] - b["min_state"]) <= 1
    assert abs(a["min_height"] - b["min_height"]) <= 1e-7 * a["min_height"]
