"""Generates tests/golden/ref_liftoff_id_vis32_256x128.npz from the
reference build in oracle/_ref (make -C oracle), for the lift-off tests.

  1. The reference's own simulation driver (fluid_test.cc) runs the
     id_vis32 physics at 256x128 with height output, writing the 251 frames
     of the run (gas_layer_solve.cc:258-282); the reference's analysis tool
     (tt_analysis.cc) reads them, smoothed and with -r. The fixture keeps the
     frames and the tool's output files and summary lines.
  2. The reference driver (oracle/ref_driver.cc, heights) writes the height
     after each of the first 1800 steps; the oracle's restatement of the
     analysis (oracle/liftoff.py) turns them into per-step minima and the
     per-step lift-off state of each mode.

    python tests/golden/make_liftoff_golden.py
"""
import glob
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import liftoff as L  # noqa: E402
from oracle import vdi_oracle as vo  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
CFG = os.path.join(HERE, "id_vis32.cfg")
STEPS = 1800


def run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, env=dict(os.environ, OMP_NUM_THREADS="8"))
    if r.returncode != 0:
        raise RuntimeError(f"{cmd}: {r.stderr}")
    return r.stdout


def main():
    text = open(CFG).read()
    P = vo.parse_cfg(text)
    out = {}
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "id32.cfg"), "w") as f:
            f.write(text + "output h\n")
        run([os.path.join(REF, "fluid_test"), "id32.cfg"], d)
        nf = len(glob.glob(os.path.join(d, "id32.odr", "height.*")))
        frames = []
        for i in range(nf):
            a = np.fromfile(os.path.join(d, "id32.odr", f"height.{i}"), dtype=np.float32)
            m = int(a[0])
            out["frames_x"] = a[1:m + 1]
            frames.append(a[m + 2:2 * m + 2])
        out["frames_h"] = np.array(frames, dtype=np.float32)
        s1 = run([os.path.join(REF, "tt_analysis"), "id32.odr"], d)
        s2 = run([os.path.join(REF, "tt_analysis"), "-r", "id32.odr"], d)
        out["tta"] = np.array(open(os.path.join(d, "id32.tta")).read())
        out["ttb"] = np.array(open(os.path.join(d, "id32.ttb")).read())
        out["summary_tta"] = np.array(s1.strip().splitlines()[-1])
        out["summary_ttb"] = np.array(s2.strip().splitlines()[-1])
        hb = os.path.join(d, "heights.bin")
        info = run([os.path.join(REF, "vdi_ref_driver"), "heights", CFG, str(STEPS), hb], d)
        dt = float(info.split('"dt": ')[1].split("}")[0])
        rows = np.fromfile(hb).reshape(-1, P.m + 1)
    x = np.array([np.float32(P.ax + (i + 0.5) * P.dx) for i in range(P.m)], dtype=np.float64)
    dx = (x[-1] - x[0]) / (P.m - 1)
    heights = [r[1:].astype(np.float32).astype(np.float64) for r in rows]
    out["dt"] = np.array(dt)
    out["step_hmax"] = np.array(max(float(np.abs(r[1:]).max()) for r in rows))
    for name, sm in (("smoothed", True), ("raw", False)):
        res, s = L.analyse(heights, x, dx, dt, P.R, P.V, P.h0, smoothed=sm)
        out[f"step_x_{name}"] = np.array([r[2] for r in res])
        out[f"step_h_{name}"] = np.array([r[3] for r in res])
        out[f"step_liftoff_{name}"] = np.array(s.gimin)
        print(name, "per-step lift-off state", s.gimin, "height", s.gfmin, "searching", s.hsearch)
    np.savez_compressed(os.path.join(HERE, "ref_liftoff_id_vis32_256x128.npz"), **out)
    print("frames", nf, "tta summary", str(out["summary_tta"]), "ttb summary", str(out["summary_ttb"]))


if __name__ == "__main__":
    main()
