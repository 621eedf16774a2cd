"""Multigrid parity on the GPU: the operators equal the reference's stencil
accessors (mgs_mac.hh:33-45, mgs_fem.cc:32-53, visco_impl.hh:36-46), and
solves reach ||b-Az||/||b|| <= rtol and agree with an exact sparse solve."""
import numpy as np
import pytest

from oracle import vdi_oracle as vo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def V():
    import vdropimpact_b200 as V
    return V


def _torch():
    import torch
    return torch


def gaussians_rhs(m, n, seed, k=64):
    """Zero-mean sum of k Gaussians (centres uniform, widths 0.01-0.1 of the
    domain, amplitudes N(0,1)): the single-projection workload's RHS."""
    from vdropimpact_b200 import projection_source
    return projection_source(m, n, seed, k)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("m,n", [(64, 32), (256, 128)])
def test_mac_apply_equals_accessors(V, m, n):
    torch = _torch()
    dx, dy = 2. / (m - 1), 2. / (n - 1)
    A = vo.mac_matrix(m, n, 1. / (dx * dx), 1. / (dy * dy))
    s = V.MgsMac(m, n, dx, dy)
    z = np.random.default_rng(1).standard_normal(m * n)
    s.z.copy_(torch.from_numpy(z))
    y = s.apply().cpu().numpy()
    assert _rel(y, A @ z) < 1e-14


@pytest.mark.parametrize("M,N", [(65, 33), (257, 129)])
def test_fem_apply_equals_accessors(V, M, N):
    torch = _torch()
    dx, dy = 1e-3, 1.3e-3
    A = vo.fem_matrix(M, N, dx, dy)
    s = V.MgsFem(M, N, dx, dy)
    z = np.random.default_rng(2).standard_normal(M * N)
    s.z.copy_(torch.from_numpy(z))
    y = s.apply().cpu().numpy()
    assert _rel(y, A @ z) < 1e-14


@pytest.mark.parametrize("x_sym,horiz", [(True, True), (True, False), (False, True)])
def test_visc_apply_equals_accessors(V, x_sym, horiz):
    torch = _torch()
    m, n, vfx, vfy = 128, 64, 0.37, 0.41
    A = vo.visco_matrix(m, n, vfx, vfy, x_sym, horiz)
    s = V.ViscoImpl(m, n, x_sym, horiz, vfx, vfy)
    z = np.random.default_rng(3).standard_normal(m * n)
    s.z.copy_(torch.from_numpy(z))
    y = s.apply().cpu().numpy()
    assert _rel(y, A @ z) < 1e-14


@pytest.mark.parametrize("prec", ["fp64", "mixed", "hybrid"])
@pytest.mark.parametrize("m,n", [(256, 128), (512, 256)])
def test_mac_solve_gaussians(V, m, n, prec):
    torch = _torch()
    dx = 1. / m
    b = gaussians_rhs(m, n, seed=7)
    A = vo.mac_matrix(m, n, 1. / (dx * dx), 1. / (dx * dx))
    s = V.MgsMac(m, n, dx, dx)
    s.b.copy_(torch.from_numpy(b))
    v, rel = s.solve_v_cycle(rtol=1e-10, precision=prec)
    z = s.z.cpu().numpy()
    r = b - A @ z
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10 * (1 + 1e-6)
    assert rel <= 1e-10
    assert 1 <= v <= 40
    zd = vo.DirectSolver(A).solve(b)
    assert _rel(z, zd) < 1e-6


@pytest.mark.parametrize("prec", ["fp64", "mixed", "hybrid"])
def test_fem_solve(V, prec):
    torch = _torch()
    M, N = 257, 129
    dx = dy = 1. / (M - 1)
    rng = np.random.default_rng(11)
    b = np.zeros((N, M))
    b[1:, :] = gaussians_rhs(M, N - 1, seed=5).reshape(N - 1, M) * dx * dx
    i = np.arange(M)
    c = vo.fem_coeffs(dx, dy)
    b[0, :] = vo.fem_a_cc(M, N, i, 0, c['fm']) * rng.uniform(100, 200, M)
    b = b.ravel()
    A = vo.fem_matrix(M, N, dx, dy)
    s = V.MgsFem(M, N, dx, dy)
    s.b.copy_(torch.from_numpy(b))
    v, rel = s.solve_v_cycle(rtol=1e-10, precision=prec)
    z = s.z.cpu().numpy()
    assert np.linalg.norm(b - A @ z) / np.linalg.norm(b) <= 1e-10 * (1 + 1e-6)
    assert v <= 40
    zd = vo.DirectSolver(A).solve(b)
    assert _rel(z, zd) < 1e-7


@pytest.mark.parametrize("x_sym,horiz", [(True, True), (True, False), (False, False)])
@pytest.mark.parametrize("prec", ["fp64", "mixed", "hybrid"])
def test_visc_solve(V, x_sym, horiz, prec):
    torch = _torch()
    m, n, vfx, vfy = 256, 128, 0.4, 0.4
    b = np.random.default_rng(13).standard_normal(m * n)
    A = vo.visco_matrix(m, n, vfx, vfy, x_sym, horiz)
    s = V.ViscoImpl(m, n, x_sym, horiz, vfx, vfy)
    s.b.copy_(torch.from_numpy(b))
    v, rel = s.solve_v_cycle(rtol=1e-10, precision=prec)
    z = s.z.cpu().numpy()
    assert np.linalg.norm(b - A @ z) / np.linalg.norm(b) <= 1e-10 * (1 + 1e-6)
    assert v <= 20
    assert _rel(z, vo.DirectSolver(A).solve(b)) < 1e-9


@pytest.mark.parametrize("prec", ["fp64", "mixed", "hybrid"])
@pytest.mark.parametrize("kind,m,n", [("mac", 64, 32), ("mac", 1024, 512), ("fem", 513, 257), ("mac", 135, 77)])
def test_zero_rhs_gives_zero(V, kind, m, n, prec):
    """A zero source is solved at once with z = 0, whatever z held, on one
    block and on many, on the fixed and the Galerkin hierarchy."""
    s = (V.MgsMac if kind == "mac" else V.MgsFem)(m, n, 0.1, 0.1)
    s.z.fill_(3.0)
    v, rel = s.solve_v_cycle(precision=prec)
    assert v == 0 and float(s.z.abs().max()) == 0.0


def test_vcycle_cap_reports_error(V):
    torch = _torch()
    m, n = 128, 64
    s = V.MgsMac(m, n, 1. / m, 1. / m)
    s.b.copy_(torch.from_numpy(gaussians_rhs(m, n, 3)))
    with pytest.raises(V.VdiError) as e:
        s.solve_v_cycle(rtol=1e-14, max_vcycles=2)
    assert e.value.status == 5


def test_nonfinite_rhs_reports_error(V):
    torch = _torch()
    s = V.MgsMac(64, 32, 0.1, 0.1)
    s.b.fill_(1.0)
    s.b[100] = float("nan")
    with pytest.raises(V.VdiError) as e:
        s.solve_v_cycle()
    assert e.value.status == 8


def test_matches_reference_dipole_solve(V, ref_driver, tmp_path):
    """mg_test's dipole source (mg_test.cc:87-91) solved by the reference
    build and by the GPU, both to a tight tolerance."""
    import os
    import subprocess
    torch = _torch()
    for kind, m, n in (("mac", 128, 64), ("fem", 129, 65)):
        dx, dy = 2. / (m - 1), 2. / (n - 1)
        b = np.zeros(m * n)
        b[m // 5 + (n // 3) * m] = 1
        b[(6 * m) // 7 + ((2 * n) // 3) * m] = -1
        if kind == "fem":
            b[:m] = 0.
        bf, zf = tmp_path / "b.bin", tmp_path / "z.bin"
        b.tofile(bf)
        env = dict(os.environ, VDI_MG_RTOL="1e-13")
        subprocess.run([ref_driver, kind, str(m), str(n), repr(dx), repr(dy), str(bf), str(zf)], check=True,
                       env=env, capture_output=True)
        zr = np.fromfile(zf)
        s = (V.MgsMac if kind == "mac" else V.MgsFem)(m, n, dx, dy)
        s.b.copy_(torch.from_numpy(b))
        s.solve_v_cycle(rtol=1e-13)
        assert _rel(s.z.cpu().numpy(), zr) < 1e-9, kind


# ----------------------------------------------------------------- any size
# Sizes the constant-stencil hierarchy cannot coarsen to a small level (an
# odd factor in a side) run on the Galerkin hierarchy; VDI_MG_GENERAL=1 forces
# it on power-of-two sizes too.

@pytest.fixture
def force_general(monkeypatch):
    monkeypatch.setenv("VDI_MG_GENERAL", "1")


@pytest.mark.parametrize("m,n", [(96, 64), (200, 100), (135, 77), (256, 128)])
def test_mac_solve_any_size(V, m, n, monkeypatch):
    torch = _torch()
    if (m, n) == (256, 128):
        monkeypatch.setenv("VDI_MG_GENERAL", "1")
    dx, dy = 2. / (m - 1), 2. / (n - 1)
    b = gaussians_rhs(m, n, seed=3)
    A = vo.mac_matrix(m, n, 1. / (dx * dx), 1. / (dy * dy))
    s = V.MgsMac(m, n, dx, dy)
    s.b.copy_(torch.from_numpy(b))
    v, rel = s.solve_v_cycle(rtol=1e-10)
    z = s.z.cpu().numpy()
    assert np.linalg.norm(b - A @ z) / np.linalg.norm(b) <= 1e-10 * (1 + 1e-6)
    assert v <= 30, v
    assert _rel(z, vo.DirectSolver(A).solve(b)) < 1e-6


@pytest.mark.parametrize("M,N", [(96, 64), (201, 101), (57, 130), (257, 129)])
def test_fem_solve_any_size(V, M, N, monkeypatch):
    torch = _torch()
    if (M, N) == (257, 129):
        monkeypatch.setenv("VDI_MG_GENERAL", "1")
    dx, dy = 1. / (M - 1), 1.2 / (N - 1)
    rng = np.random.default_rng(17)
    b = np.zeros((N, M))
    b[1:, :] = rng.standard_normal((N - 1, M)) * dx * dy
    c = vo.fem_coeffs(dx, dy)
    b[0, :] = vo.fem_a_cc(M, N, np.arange(M), 0, c['fm']) * rng.uniform(1, 2, M)
    b = b.ravel()
    A = vo.fem_matrix(M, N, dx, dy)
    s = V.MgsFem(M, N, dx, dy)
    s.b.copy_(torch.from_numpy(b))
    v, rel = s.solve_v_cycle(rtol=1e-10)
    z = s.z.cpu().numpy()
    assert np.linalg.norm(b - A @ z) / np.linalg.norm(b) <= 1e-10 * (1 + 1e-6)
    assert v <= 30, v
    assert _rel(z, vo.DirectSolver(A).solve(b)) < 1e-7


@pytest.mark.parametrize("x_sym,horiz", [(True, True), (False, False)])
@pytest.mark.parametrize("vf", [0.4, 40.0])
def test_visc_solve_any_size(V, x_sym, horiz, vf):
    torch = _torch()
    m, n = 200, 100
    b = np.random.default_rng(19).standard_normal(m * n)
    A = vo.visco_matrix(m, n, vf, vf, x_sym, horiz)
    s = V.ViscoImpl(m, n, x_sym, horiz, vf, vf)
    s.b.copy_(torch.from_numpy(b))
    v, rel = s.solve_v_cycle(rtol=1e-10)
    z = s.z.cpu().numpy()
    assert np.linalg.norm(b - A @ z) / np.linalg.norm(b) <= 1e-10 * (1 + 1e-6)
    assert v <= 30, v
    assert _rel(z, vo.DirectSolver(A).solve(b)) < 1e-9


def test_general_vcycle_count_comparable(V, monkeypatch):
    """On a power-of-two grid the general hierarchy converges in about as many
    V-cycles as the constant-stencil one."""
    torch = _torch()
    m, n = 256, 128
    dx = 1. / m
    b = torch.from_numpy(gaussians_rhs(m, n, seed=9))
    s = V.MgsMac(m, n, dx, dx)
    s.b.copy_(b)
    v_fast, _ = s.solve_v_cycle(rtol=1e-10)
    monkeypatch.setenv("VDI_MG_GENERAL", "1")
    g = V.MgsMac(m, n, dx, dx)
    g.b.copy_(b)
    v_gen, _ = g.solve_v_cycle(rtol=1e-10)
    assert v_gen <= v_fast + 4, (v_gen, v_fast)


# ------------------------------------------------------- pure Neumann
def _neumann_exact(m, n, dx, dy, b):
    """The zero-mean solution of the singular system, from the bordered
    matrix [[A, 1], [1^T, 0]] and the projected source."""
    import scipy.sparse as sp
    A = sp.csr_matrix(vo.mac_matrix(m, n, 1. / (dx * dx), 1. / (dy * dy), neumann_bottom=True))
    one = sp.csr_matrix(np.ones((m * n, 1)))
    K = sp.bmat([[A, one], [one.T, None]]).tocsc()
    rhs = np.concatenate([b - b.mean(), [0.]])
    return vo.DirectSolver(K).solve(rhs)[:-1], A


@pytest.mark.parametrize("m,n", [(256, 128), (512, 256), (200, 100)])
def test_mac_neumann_matches_exact(V, m, n):
    """The source is given a nonzero mean on purpose: the solve projects it
    out (the compatibility reduction) and returns the zero-mean solution."""
    torch = _torch()
    dx = 1. / m
    b = gaussians_rhs(m, n, seed=21) + 0.37
    zx, A = _neumann_exact(m, n, dx, dx, b)
    s = V.MgsMacNeumann(m, n, dx, dx)
    s.b.copy_(torch.from_numpy(b))
    v, rel = s.solve_v_cycle(rtol=1e-10)
    z = s.z.cpu().numpy()
    bp = b - b.mean()
    assert np.linalg.norm(bp - A @ z) / np.linalg.norm(bp) <= 1e-10 * (1 + 1e-6)
    assert abs(z.mean()) <= 1e-12 * np.abs(z).max()
    assert v <= 30, v
    assert _rel(z, zx) < 1e-7


def test_mac_neumann_config2_size(V):
    """2048x1024, the single-projection workload's size: residual of the
    projected source and the zero mean, checked on the device."""
    torch = _torch()
    m, n = 2048, 1024
    dx = 1. / m
    b = torch.from_numpy(gaussians_rhs(m, n, seed=5) + 1.5).cuda()
    s = V.MgsMacNeumann(m, n, dx, dx)
    s.b.copy_(b)
    v, rel = s.solve_v_cycle(rtol=1e-10)
    bp = b - b.mean()
    r = bp - s.apply()
    assert float(torch.linalg.norm(r) / torch.linalg.norm(bp)) <= 1e-10 * (1 + 1e-6)
    assert abs(float(s.z.mean())) <= 1e-12 * float(s.z.abs().max())
    assert v <= 30, v


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_repeated_solves_replay_the_same_solve(V, prec):
    """The second and later solves of the same arrays run from a captured
    graph (one launch, one status read): the same kernels in the same order
    as the first, host-driven solve, so the same iterate bit for bit and the
    same V-cycle count; a changed tolerance and the V-cycle cap still
    apply."""
    torch = _torch()
    m, n = 256, 128
    dx = 1. / m
    b = torch.from_numpy(gaussians_rhs(m, n, seed=13)).cuda()
    s = V.MgsMac(m, n, dx, 1.5 * dx)
    s.b.copy_(b)
    runs = []
    for _ in range(3):
        s.z.zero_()
        runs.append((s.solve_v_cycle(rtol=1e-10, precision=prec), s.z.clone()))
    (v0, _), z0 = runs[0]
    for (v, _), z in runs[1:]:
        assert v == v0
        assert torch.equal(z, z0)
    s.z.zero_()
    v8, rel8 = s.solve_v_cycle(rtol=1e-8, precision=prec)
    assert rel8 <= 1e-8 and v8 < v0
    s.z.zero_()
    with pytest.raises(V.VdiError):
        s.solve_v_cycle(rtol=1e-10, max_vcycles=1, precision=prec)
