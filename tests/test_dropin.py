"""The C++ drop-in classes (vdropimpact_b200/host): the reference's own
drivers fluid_test.cc, mg_test.cc and tri_test.cc, compiled unmodified
against them (oracle/Makefile, target b200), run on the GPU beside the same
drivers built on the reference's classes (oracle/_ref), and their output
files are compared: every frame format (Gnuplot float32 matrices and
profiles, the full-precision profiles), the restart files, and a run resumed
on the GPU from a restart file the CPU reference wrote.

Float32 outputs agree to float rounding of values that agree within 1e-8 of
each field's scale; double outputs within 1e-8 of the scale."""
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF = os.path.join(ROOT, "oracle", "_ref")
LIB = os.path.join(ROOT, "vdropimpact_b200", "_lib")
OUTPUTS = "u v p pb pbfull w h fbd pg hfull fbdfull pgfull"


def _cfg(frames=10, t_end_nd=2.0, restart=5):
    lines = [l for l in open(os.path.join(HERE, "golden", "id_vis32.cfg")).read().splitlines()
             if not l.split("#")[0].strip().startswith(("t_end_nd", "frames"))]
    return "\n".join(lines + [f"t_end_nd {t_end_nd}", f"frames {frames}", f"output {OUTPUTS}",
                              f"restart_freq {restart}"]) + "\n"


def _need(*names):
    for n in names:
        if not os.path.exists(os.path.join(REF, n)):
            pytest.skip(f"oracle/_ref/{n} not built (make -C oracle all b200)")


def _run(cmd, cwd, ok=True):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 4)))
    if ok and r.returncode != 0:
        raise AssertionError(f"{cmd} failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    return r


def test_host_library_and_driver_built():
    assert os.path.exists(os.path.join(LIB, "libvdi_host.so"))
    assert os.path.exists(os.path.join(LIB, "vdi_fluid_test"))


@pytest.mark.parametrize("extra,msg", [("gas_layer_data 64 64 p.dat t.dat", "outside the GPU path"),
                                       ("frobnicate 1", "Keyword 'frobnicate' not understood"),
                                       ("output h bogus", "Output type not understood")])
def test_config_errors_exit_like_the_reference(tmp_path, extra, msg):
    """fileinfo's checks (fileinfo.cc:56-129) end the run with exit status 1
    and a message, before any device work."""
    cfg = tmp_path / "bad.cfg"
    cfg.write_text(_cfg() + extra + "\n")
    r = _run([os.path.join(LIB, "vdi_fluid_test"), str(cfg)], str(tmp_path), ok=False)
    assert r.returncode == 1 and msg in r.stderr, r.stderr


def _gp(path):
    """A Gnuplot binary matrix: (x, rows of (y, values))."""
    a = np.fromfile(path, dtype=np.float32)
    n = int(a[0])
    a = a.reshape(-1, n + 1)
    return a[0, 1:], a[1:, 0], a[1:, 1:]


def _full(path):
    """A full-precision profile: int l, double ax, bx, l doubles."""
    raw = open(path, "rb").read()
    l = int(np.frombuffer(raw[:4], dtype=np.int32)[0])
    v = np.frombuffer(raw[4:], dtype=np.float64)
    return l, v[:2], v[2:]


def _compare_frame(a_dir, b_dir, k):
    for name in ("u", "v", "p", "pb", "w", "height", "fbd", "pg"):
        xa, ya, fa = _gp(os.path.join(a_dir, f"{name}.{k}"))
        xb, yb, fb = _gp(os.path.join(b_dir, f"{name}.{k}"))
        assert np.array_equal(xa, xb) and np.array_equal(ya, yb), name
        scale = max(float(np.abs(fb).max()), 1e-300)
        assert np.abs(fa.astype(np.float64) - fb).max() <= 1e-8 * scale + 2 ** -23 * np.abs(fb).max(), (name, k)
    for name in ("hfull", "fbdfull", "pgfull", "pbfull"):
        la, ha, va = _full(os.path.join(a_dir, f"{name}.{k}"))
        lb, hb, vb = _full(os.path.join(b_dir, f"{name}.{k}"))
        assert la == lb and np.array_equal(ha, hb) and va.size == vb.size, name
        scale = max(float(np.abs(vb).max()), 1e-300)
        assert np.abs(va - vb).max() <= 1e-8 * scale, (name, k)


def _restart_parts(path, m, n, nt=0):
    """The record of fluid_2d_sio.cc:97-119 and gas_layer_solve.cc:323-331:
    time; u, v, p interleaved over the ghosted grid; the 2*nt tracer
    coordinates; Vframe; the gas layer's p[m+1], tau[2..m+1], h[m], ht[m],
    pg[m+1]."""
    r = np.fromfile(path)
    ng = (m + 4) * (n + 4)
    assert r.size == 1 + 3 * ng + 2 * nt + 1 + (m + 1) + 3 * m + (m + 1)
    f = r[1:1 + 3 * ng].reshape(ng, 3)
    o = 1 + 3 * ng
    parts = {"time": r[:1], "u": f[:, 0], "v": f[:, 1], "p": f[:, 2]}
    if nt:
        parts["tm"] = r[o:o + 2 * nt]
        o += 2 * nt
    parts["Vframe"] = r[o:o + 1]
    o += 1
    for k, l in (("gp", m + 1), ("tau", m), ("h", m), ("ht", m), ("pg", m + 1)):
        parts[k] = r[o:o + l]
        o += l
    return parts


def _compare_restart(a, b, m=256, n=128, nt=0, tol=1e-8):
    pa, pb = _restart_parts(a, m, n, nt), _restart_parts(b, m, n, nt)
    assert pa["time"][0] == pb["time"][0]
    for k in pb:
        scale = max(float(np.abs(pb[k]).max()), 1e-300)
        assert np.abs(pa[k] - pb[k]).max() <= tol * scale, k


@pytest.mark.gpu
def test_tri_test_matches_reference(tmp_path):
    _need("tri_test", "tri_test_b200")
    a = _run([os.path.join(REF, "tri_test_b200")], str(tmp_path)).stdout.split()
    b = _run([os.path.join(REF, "tri_test")], str(tmp_path)).stdout.split()
    assert len(a) == len(b)
    assert np.allclose(np.array(a, float), np.array(b, float), rtol=1e-5, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["0", "2"])
def test_mg_test_matches_reference(tmp_path, case):
    _need("mg_test", "mg_test_b200")
    da, db = tmp_path / "b200", tmp_path / "ref"
    da.mkdir()
    db.mkdir()
    _run([os.path.join(REF, "mg_test_b200"), case, "96", "64"], str(da))
    _run([os.path.join(REF, "mg_test"), case, "96", "64"], str(db))
    for f in ("b.0", "z.0"):
        xa, ya, fa = _gp(str(da / f))
        xb, yb, fb = _gp(str(db / f))
        assert np.array_equal(xa, xb) and np.array_equal(ya, yb)
        assert np.abs(fa.astype(np.float64) - fb).max() <= 1e-7 * np.abs(fb).max(), f
    _, _, ra = _gp(str(da / "r.0"))
    _, _, ba = _gp(str(da / "b.0"))
    assert np.linalg.norm(ra) <= 1e-9 * np.linalg.norm(ba)


@pytest.mark.gpu
def test_fluid_test_frames_and_restarts_match_reference(tmp_path):
    _need("fluid_test", "fluid_test_b200")
    da, db = tmp_path / "b200", tmp_path / "ref"
    for d in (da, db):
        d.mkdir()
        (d / "run.cfg").write_text(_cfg())
    _run([os.path.join(REF, "fluid_test_b200"), "run.cfg"], str(da))
    _run([os.path.join(REF, "fluid_test"), "run.cfg"], str(db))
    for k in range(11):
        _compare_frame(str(da / "run.odr"), str(db / "run.odr"), k)
    for k in (5, 10):
        _compare_restart(str(da / "run.odr" / f"res.{k}"), str(db / "run.odr" / f"res.{k}"))


@pytest.mark.gpu
def test_fluid_test_tracers_and_moving_frame_match_reference(tmp_path):
    """fluid_test with 40 tracers and the nif_center frame: the trace.N
    frames (fluid_2d_sio.cc:121-145), every field frame and the restart
    records (which carry the tracers) agree with the reference's. Both
    processes draw the tracers with rand() from its initial state. The
    frame velocity, taken from four cells each step and subtracted from all
    of v, carries each step's solver differences (both sides stop at a
    1e-10 residual) into the next, so over this run's frames the restart
    records are held to 1e-7 of each field's scale (the 50-step
    comparisons in test_gpu_step hold 1e-8)."""
    _need("fluid_test", "fluid_test_b200")
    da, db = tmp_path / "b200", tmp_path / "ref"
    txt = _cfg() + "tracers 40\nnif_center\n"
    for d in (da, db):
        d.mkdir()
        (d / "run.cfg").write_text(txt)
    _run([os.path.join(REF, "fluid_test_b200"), "run.cfg"], str(da))
    _run([os.path.join(REF, "fluid_test"), "run.cfg"], str(db))
    for k in range(11):
        _compare_frame(str(da / "run.odr"), str(db / "run.odr"), k)
        ta = np.fromfile(str(da / "run.odr" / f"trace.{k}"), dtype=np.float32)
        tb = np.fromfile(str(db / "run.odr" / f"trace.{k}"), dtype=np.float32)
        assert ta.size == tb.size == 80
        assert np.abs(ta.astype(np.float64) - tb).max() <= 2 ** -22 * np.abs(tb).max(), k
    for k in (5, 10):
        _compare_restart(str(da / "run.odr" / f"res.{k}"), str(db / "run.odr" / f"res.{k}"), nt=40, tol=1e-7)
    vf = _restart_parts(str(db / "run.odr" / "res.10"), 256, 128, 40)["Vframe"][0]
    assert vf < 0.45   # the frame followed the drop


@pytest.mark.gpu
def test_resume_on_gpu_from_reference_restart(tmp_path):
    """The GPU driver (our own, vdi_fluid_test -r) resumes from res.5 written
    by the CPU reference and writes the frames 6-10 that the reference,
    resumed from the same file, writes. (The boundary flux fbd accumulates
    over a run and is not part of the restart record, gas_layer_solve.cc:157,
    323-331, so a resumed run is compared with a resumed run.)"""
    _need("fluid_test")
    db = tmp_path / "ref"
    db.mkdir()
    (db / "run.cfg").write_text(_cfg())
    _run([os.path.join(REF, "fluid_test"), "run.cfg"], str(db))
    runs = {}
    for name, exe in (("gpu", os.path.join(LIB, "vdi_fluid_test")), ("cpu", os.path.join(REF, "fluid_test"))):
        d = tmp_path / name
        d.mkdir()
        (d / "run.cfg").write_text(_cfg())
        (d / "run.odr").mkdir()
        shutil.copy(db / "run.odr" / "res.5", d / "run.odr" / "res.5")
        r = _run([exe, "-r", "run.cfg"], str(d))
        assert "Starting from restart file at frame 5" in r.stdout
        runs[name] = d / "run.odr"
    for k in range(6, 11):
        _compare_frame(str(runs["gpu"]), str(runs["cpu"]), k)
    _compare_restart(str(runs["gpu"] / "res.10"), str(runs["cpu"] / "res.10"))
