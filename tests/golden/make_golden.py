"""Generates the golden fixtures of tests/golden from the reference's own code
(built by oracle/Makefile into oracle/_ref from the reference sources).

    make -C oracle && python tests/golden/make_golden.py

Fixtures:
  ref_id_vis32_256x128.npz  the 256x128 initial-deceleration case run by the
      reference for 200 steps (multigrid solves to relative residual 1e-13):
      for steps 0, 1, 50 and 200 the gas-layer arrays in full and u, v, p on
      every 4th row and column of the ghosted grid, plus whole-field sums,
      sums of squares and maxima.
  ref_dipole_mg.npz  mg_test's dipole source (mg_test.cc:87-91) solved by the
      reference's mgs_mac (128x64) and mgs_fem (129x65) to 1e-13, every 2nd
      row and column.
  ref_tracers_frame_256x128.npz  the 256x128 case with tracers and the
      nif_center non-inertial frame, with and without x_sym, run by the
      reference for 50 steps: per step the time, Vframe and the tracer
      positions (the first row holds the positions init_tracers drew with
      rand()), and the step-50 summary as above. (nif_range is
      not generated: the reference computes its window from fileinfo::xsp,
      which no constructor sets, fileinfo.cc:182-186, so its result depends
      on uninitialised memory.)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import vdi_oracle as vo  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "vdi_ref_driver")
STEPS = (0, 1, 50, 200)
# cases of the tracer / non-inertial-frame fixture: extra .cfg lines, and
# whether x_sym stays
FRAME_CASES = {
    "center": ("tracers 64\nnif_center\n", True),
    "center_full": ("tracers 32\nnif_center\n", False),
}
FRAME_STEPS = 50


def frame_cfg(case):
    extra, xsym = FRAME_CASES[case]
    lines = [l for l in open(os.path.join(HERE, "id_vis32.cfg")).read().splitlines()
             if l.split("#")[0].strip() not in ("tracers",) and not l.split("#")[0].strip().startswith("tracers")
             and (xsym or l.split("#")[0].strip() != "x_sym")]
    return "\n".join(lines) + "\n" + extra


def summarize(st):
    out = {}
    for k in ("u", "v", "p"):
        a = st[k]
        out[k + "_sub"] = a[::4, ::4].copy()
        out[k + "_sum"] = np.array(a.sum())
        out[k + "_sumsq"] = np.array((a * a).sum())
        out[k + "_max"] = np.array(np.abs(a).max())
    for k in ("gp", "tau", "h", "fbd", "pg", "ht"):
        out[k] = st[k]
    out["time"] = np.array(st["time"])
    return out


def main():
    env = dict(os.environ, VDI_MG_RTOL="1e-13")
    with tempfile.TemporaryDirectory() as td:
        cfg = os.path.join(HERE, "id_vis32.cfg")
        out = os.path.join(td, "s.bin")
        subprocess.run([DRIVER, "dump", cfg, str(max(STEPS)), "1", out], check=True, env=env)
        states = vo.read_states(out)
        data = {}
        for k in STEPS:
            for key, val in summarize(states[k]).items():
                data[f"s{k}_{key}"] = val
        np.savez_compressed(os.path.join(HERE, "ref_id_vis32_256x128.npz"), **data)

        dip = {}
        for kind, m, n in (("mac", 128, 64), ("fem", 129, 65)):
            dx, dy = 2. / (m - 1), 2. / (n - 1)
            b = np.zeros(m * n)
            b[m // 5 + (n // 3) * m] = 1
            b[(6 * m) // 7 + ((2 * n) // 3) * m] = -1
            bf, zf = os.path.join(td, "b.bin"), os.path.join(td, "z.bin")
            b.tofile(bf)
            subprocess.run([DRIVER, kind, str(m), str(n), repr(dx), repr(dy), bf, zf], check=True, env=env,
                           capture_output=True)
            dip[f"{kind}_z_sub"] = np.fromfile(zf).reshape(n, m)[::2, ::2].copy()
            dip[f"{kind}_dims"] = np.array([m, n, dx, dy])
        np.savez_compressed(os.path.join(HERE, "ref_dipole_mg.npz"), **dip)

        fr = {}
        for case in FRAME_CASES:
            cfg = os.path.join(td, f"{case}.cfg")
            open(cfg, "w").write(frame_cfg(case))
            tr = os.path.join(td, f"{case}.trace")
            subprocess.run([DRIVER, "tracers", cfg, str(FRAME_STEPS), tr], check=True, env=env, capture_output=True)
            raw = np.fromfile(tr)
            fr[f"{case}_trace"] = raw.reshape(FRAME_STEPS + 1, -1)
            out = os.path.join(td, f"{case}.bin")
            subprocess.run([DRIVER, "dump", cfg, str(FRAME_STEPS), "1", out], check=True, env=env,
                           capture_output=True)
            states = vo.read_states(out)
            for k in (FRAME_STEPS,):
                for key, val in summarize(states[k]).items():
                    fr[f"{case}_s{k}_{key}"] = val
                fr[f"{case}_s{k}_Vframe"] = np.array(states[k]["Vframe"])
            fr[f"{case}_cfg"] = np.array(frame_cfg(case))
        np.savez_compressed(os.path.join(HERE, "ref_tracers_frame_256x128.npz"), **fr)


if __name__ == "__main__":
    main()
