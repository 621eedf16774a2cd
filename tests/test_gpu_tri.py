"""Tridiagonal solver parity on the GPU against the dgtsv restatement and the
known answer of the reference's tri_test (tri_test.cc:6-30)."""
import numpy as np
import pytest

from oracle import vdi_oracle as vo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def V():
    import vdropimpact_b200 as V
    return V


def _solve(V, a, b, c, d):
    t = V.TriSolve(len(b))
    t.a[:], t.b[:], t.c[:], t.d[:] = a, b, c, d
    x = t.solve_lapack()
    return x, t.pivoted


def test_tri_test_poisson_known_answer(V):
    """u''=1 on [0,1], zero Dirichlet, 32 points: exactly x(x-1)/2."""
    m = 32
    dx = 1. / (m + 1.)
    xxsp = 1 / dx / dx
    a = np.full(m, xxsp); c = np.full(m, xxsp); b = np.full(m, -2 * xxsp); d = np.ones(m)
    x, piv = _solve(V, a, b, c, d)
    xs = (np.arange(m) + 1) * dx
    assert not piv
    np.testing.assert_allclose(x, xs * (xs - 1) / 2, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("n", [3, 7, 257, 1000, 2049])
def test_dominant_systems_use_cyclic_reduction(V, n):
    rng = np.random.default_rng(n)
    a = rng.uniform(-1, 1, n); c = rng.uniform(-1, 1, n)
    b = (np.abs(a) + np.abs(c) + rng.uniform(0.1, 1, n)) * rng.choice([-1, 1], n)
    d = rng.standard_normal(n)
    x, piv = _solve(V, a, b, c, d)
    xr, info = vo.dgtsv(a[1:], b, c[:-1], d)
    assert info == 0 and not piv
    np.testing.assert_allclose(x, xr, rtol=1e-12, atol=1e-14 * np.abs(xr).max())


@pytest.mark.parametrize("n", [5, 64, 2049])
def test_pivoting_fallback(V, n):
    rng = np.random.default_rng(100 + n)
    a = rng.uniform(-2, 2, n); c = rng.uniform(-2, 2, n); b = rng.uniform(-0.5, 0.5, n)
    d = rng.standard_normal(n)
    x, piv = _solve(V, a, b, c, d)
    xr, info = vo.dgtsv(a[1:], b, c[:-1], d)
    assert info == 0 and piv
    np.testing.assert_allclose(x, xr, rtol=1e-9, atol=1e-12 * np.abs(xr).max())


def test_singular_reports_error(V):
    n = 4
    a = np.zeros(n); b = np.zeros(n); c = np.zeros(n); d = np.ones(n)
    with pytest.raises(V.VdiError) as e:
        _solve(V, a, b, c, d)
    assert e.value.status == 7


def test_newton_system_of_config1(V):
    """The gas layer's Newton matrix (gas_layer_solve.cc:67-126) of the
    256x128 workload after a few steps, solved on the GPU."""
    import os
    cfg = os.path.join(os.path.dirname(__file__), "golden", "id_vis32.cfg")
    o = vo.Oracle(vo.parse_cfg(open(cfg).read()))
    o.init_fields()
    dt = o.prm.frame_dt()
    for _ in range(3):
        o.step(dt)
    o.gp_old[:] = o.gp; o.tau_old[:] = o.tau
    o.update_height(dt)
    o.pg_old[:] = o.pg
    a, b, c, d, _ = o.newton_assemble(1. / dt)
    x, piv = _solve(V, a, b, c, d)
    xr, info = vo.dgtsv(a[1:], b, c[:-1], d)
    np.testing.assert_allclose(x, xr, rtol=1e-11, atol=1e-13 * np.abs(xr).max())
