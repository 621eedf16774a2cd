"""CPU tests of the oracle: the numpy restatement of the step against the
reference's own code (golden fixtures made by tests/golden/make_golden.py, and
the reference build itself when oracle/_ref exists), the dgtsv restatement
against LAPACK, and tri_test's known answer (tri_test.cc:6-30)."""
import os
import subprocess

import numpy as np
import pytest
from scipy.linalg import lapack

from oracle import vdi_oracle as vo

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _cfg(m, n, drop=()):
    lines = [l for l in open(os.path.join(GOLD, "id_vis32.cfg")).read().splitlines()
             if l.split("#")[0].strip() not in drop and not l.startswith("grid_points")]
    return "\n".join(lines + [f"grid_points {m} {n}"]) + "\n"


def test_restatement_matches_reference_golden_256x128():
    """200 steps of the 256x128 initial-deceleration case against the
    reference run stored in ref_id_vis32_256x128.npz."""
    g = np.load(os.path.join(GOLD, "ref_id_vis32_256x128.npz"))
    o = vo.Oracle(vo.parse_cfg(open(os.path.join(GOLD, "id_vis32.cfg")).read()))
    o.init_fields()
    dt = o.prm.frame_dt()
    for k in range(0, 201):
        if k > 0:
            o.step(dt)
        if k in (0, 1, 50, 200):
            st = o.state()
            for f in ("u", "v", "p"):
                assert _rel(st[f][::4, ::4], g[f"s{k}_{f}_sub"]) < 1e-10, (k, f)
                np.testing.assert_allclose((st[f] * st[f]).sum(), g[f"s{k}_{f}_sumsq"], rtol=1e-10)
            for f in ("h", "pg", "gp", "tau", "fbd", "ht"):
                assert _rel(st[f], g[f"s{k}_{f}"]) < 1e-10, (k, f)
            assert st["time"] == pytest.approx(float(g[f"s{k}_time"]), rel=1e-15)


FRAME = os.path.join(GOLD, "ref_tracers_frame_256x128.npz")


@pytest.mark.parametrize("case", ["center", "center_full"])
def test_tracers_and_frame_restatement_matches_reference_golden(case):
    """50 steps with tracers (fluid_2d.cc:507-526) and the nif_center
    non-inertial frame (fluid_2d_sio.cc:228-253), with and without x_sym,
    against the reference run stored in ref_tracers_frame_256x128.npz: the
    tracer positions and Vframe after every step, the fields after 50."""
    g = np.load(FRAME)
    tr = g[f"{case}_trace"]
    o = vo.Oracle(vo.parse_cfg(str(g[f"{case}_cfg"])))
    o.init_fields()
    o.tm[:] = tr[0, 2:]
    dt = o.prm.frame_dt()
    span = max(o.prm.bx - o.prm.ax, o.prm.by - o.prm.ay)
    for k in range(1, tr.shape[0]):
        o.step(dt)
        assert o.Vframe == pytest.approx(tr[k, 1], rel=1e-12), k
        assert np.max(np.abs(o.tm - tr[k, 2:])) <= 1e-13 * span, k
    st = o.state()
    for f in ("u", "v", "p"):
        assert _rel(st[f][::4, ::4], g[f"{case}_s50_{f}_sub"]) < 1e-10, f
    for f in ("h", "pg", "gp", "tau", "fbd", "ht"):
        assert _rel(st[f], g[f"{case}_s50_{f}"]) < 1e-10, f
    assert st["Vframe"] == pytest.approx(float(g[f"{case}_s50_Vframe"]), rel=1e-12)
    # the frame moved: Vframe fell from V
    assert tr[-1, 1] < tr[0, 1] - 1e-3


def test_tracer_seeding_is_the_references_rand_sequence(tmp_path):
    """init_tracers draws the positions with the C library's rand()
    (fluid_2d.cc:495-502): a process that has not called rand() before
    reproduces the reference's positions exactly."""
    import sys
    g = np.load(FRAME)
    cfg = tmp_path / "c.cfg"
    cfg.write_text(str(g["center_cfg"]))
    out = tmp_path / "tm.npy"
    code = ("import sys, numpy as np; sys.path.insert(0, sys.argv[3]); from oracle import vdi_oracle as vo; "
            "o = vo.Oracle(vo.parse_cfg(open(sys.argv[1]).read())); o.init_fields(); np.save(sys.argv[2], o.tm)")
    subprocess.run([sys.executable, "-c", code, str(cfg), str(out), os.path.dirname(HERE)], check=True)
    assert np.array_equal(np.load(out), g["center_trace"][0, 2:])


def test_init_fields_equals_reference_exactly():
    g = np.load(os.path.join(GOLD, "ref_id_vis32_256x128.npz"))
    o = vo.Oracle(vo.parse_cfg(open(os.path.join(GOLD, "id_vis32.cfg")).read()))
    o.init_fields()
    st = o.state()
    for f in ("h", "gp", "tau", "pg", "fbd", "ht"):
        assert np.array_equal(st[f], g[f"s0_{f}"]), f
    for f in ("u", "v", "p"):
        assert np.array_equal(st[f][::4, ::4], g[f"s0_{f}_sub"]), f


@pytest.mark.parametrize("drop", [(), ("x_sym",), ("implicit_visc",), ("x_sym", "implicit_visc")])
def test_restatement_matches_reference_build(ref_driver, tmp_path, drop):
    """Both branches of x_sym and implicit_visc, 6 steps at 64x32, against the
    reference build run live (multigrid to 1e-13)."""
    txt = _cfg(64, 32, drop)
    cfg = tmp_path / "t.cfg"
    cfg.write_text(txt)
    out = tmp_path / "t.bin"
    subprocess.run([ref_driver, "dump", str(cfg), "6", "1", str(out)], check=True, capture_output=True,
                   env=dict(os.environ, VDI_MG_RTOL="1e-13"))
    refs = vo.read_states(str(out))
    o = vo.Oracle(vo.parse_cfg(txt))
    o.init_fields()
    dt = o.prm.frame_dt()
    for k in range(1, 7):
        o.step(dt)
        st = o.state()
        for f in ("u", "v", "p", "h", "pg", "gp", "tau", "fbd"):
            assert _rel(st[f], refs[k][f]) < 1e-10, (k, f)


def test_mac_fem_operators_reproduce_reference_solves():
    """The restated operator matrices solve mg_test's dipole problem to the
    reference's solution."""
    d = np.load(os.path.join(GOLD, "ref_dipole_mg.npz"))
    for kind in ("mac", "fem"):
        m, n, dx, dy = d[f"{kind}_dims"]
        m, n = int(m), int(n)
        b = np.zeros(m * n)
        b[m // 5 + (n // 3) * m] = 1
        b[(6 * m) // 7 + ((2 * n) // 3) * m] = -1
        A = vo.mac_matrix(m, n, 1. / (dx * dx), 1. / (dy * dy)) if kind == "mac" else vo.fem_matrix(m, n, dx, dy)
        z = vo.DirectSolver(A).solve(b).reshape(n, m)
        assert _rel(z[::2, ::2], d[f"{kind}_z_sub"]) < 1e-9, kind


@pytest.mark.parametrize("n", [2, 5, 64, 2049])
@pytest.mark.parametrize("pivot", [False, True])
def test_dgtsv_restatement_matches_lapack(n, pivot):
    rng = np.random.default_rng(n + 7 * pivot)
    dl = rng.uniform(-2, 2, n - 1)
    du = rng.uniform(-2, 2, n - 1)
    d = rng.uniform(-0.5, 0.5, n) if pivot else np.abs(np.r_[0, dl]) + np.abs(np.r_[du, 0]) + 1
    b = rng.standard_normal(n)
    x, info = vo.dgtsv(dl, d, du, b)
    _, _, _, xl, infol = lapack.dgtsv(dl, d, du, b)
    assert info == infol == 0
    np.testing.assert_allclose(x, xl, rtol=1e-10, atol=1e-12 * np.abs(xl).max())


def test_thomas_known_answer_tri_test():
    """tri_test.cc: u''=1 on 32 points with zero Dirichlet ends is x(x-1)/2."""
    m = 32
    dx = 1. / (m + 1.)
    xxsp = 1 / dx / dx
    x = vo.thomas(np.full(m, xxsp), np.full(m, -2 * xxsp), np.full(m, xxsp), np.ones(m))
    xs = (np.arange(m) + 1) * dx
    np.testing.assert_allclose(x, xs * (xs - 1) / 2, rtol=1e-12)


def test_reference_tri_test_binary(ref_driver):
    exe = os.path.join(os.path.dirname(ref_driver), "tri_test")
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    vals = np.array(out, dtype=float).reshape(-1, 2)
    np.testing.assert_allclose(vals[:, 1], vals[:, 0] * (vals[:, 0] - 1) / 2, atol=1e-6)


def test_newton_threshold_constants():
    """gas_layer_solve.hh:11-18."""
    assert vo.NEWTON_THRESH == (np.finfo(float).eps * 1e8) ** 2
    assert vo.MAX_NEWTON_STEPS == 256


@pytest.mark.parametrize("m,n", [(64, 32), (128, 128), (96, 40)])
def test_mac_direct_solve_matches_sparse_lu(m, n):
    """The separable exact MAC solve (the yardstick of the full-size
    single-projection test) equals a sparse LU solve of mac_matrix."""
    rng = np.random.default_rng(m + n)
    b = rng.standard_normal(m * n)
    xxsp, yysp = float(m * m), 2.25 * m * m
    A = vo.mac_matrix(m, n, xxsp, yysp)
    z = vo.mac_direct_solve(m, n, xxsp, yysp, b)
    assert _rel(z, vo.DirectSolver(A).solve(b)) < 1e-12
