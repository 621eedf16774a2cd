"""The separable exact coarse solve (cosine transforms in x, one tridiagonal
solve per mode in y) against the coarse paths it replaces: the cluster
cycle of the MAC system and the dense-inverse or single-CTA cycle of the
FEM system (VDI_MG_FAST_COARSE=0 restores those).

The transform solve is exact on its level, where the other paths run one
V-cycle of the coarser levels, so a solve may take fewer V-cycles; both
reach the 1e-10 residual, and their solutions agree within what that
residual leaves (1e-8 of the solution's scale)."""
import numpy as np
import pytest

from test_gpu_mg import gaussians_rhs, _rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def V():
    import vdropimpact_b200 as V
    return V


def _make(V, kind, m, n, fast, monkeypatch):
    monkeypatch.setenv("VDI_MG_FAST_COARSE", "1" if fast else "0")
    if kind == "mac":
        dx = 1.0 / m
        s = V.MgsMac(m, n, dx, 1.5 * dx)
    else:
        s = V.MgsFem(m, n, 1.0 / (m - 1), 1.5 / (m - 1))
    monkeypatch.delenv("VDI_MG_FAST_COARSE")
    return s


def _source(kind, m, n, seed):
    import torch
    if kind == "mac":
        return torch.from_numpy(gaussians_rhs(m, n, seed=seed))
    g = torch.Generator().manual_seed(seed)
    b = torch.randn(m * n, dtype=torch.float64, generator=g)
    b[:m] = 0.3
    return b


# (kind, m, n, level solved by transforms): 256x128 for the MAC grids from
# 2048x1024, 257x129 for the FEM grids from 2049x1025; the first level of at
# most 40000 unknowns on the others
CASES = [("mac", 2048, 1024, 3), ("mac", 512, 256, 1), ("mac", 96, 32, 1), ("mac", 1024, 512, 2),
         ("fem", 2049, 1025, 3), ("fem", 513, 257, 1), ("fem", 129, 65, 1), ("fem", 641, 385, 2)]


@pytest.mark.parametrize("prec", ["fp64", "mixed", "hybrid"])
@pytest.mark.parametrize("kind,m,n,lev", CASES)
def test_transform_coarse_solve_matches_other_paths(V, kind, m, n, lev, prec, monkeypatch):
    b = _source(kind, m, n, seed=7)
    res = {}
    for fast in (True, False):
        s = _make(V, kind, m, n, fast, monkeypatch)
        first, ctas = s.coarse_cycle(precision=prec if prec == "mixed" else None)
        if fast:
            assert (first, ctas) == (lev, -1)
        else:
            assert ctas != -1
        s.b.copy_(b)
        s.z.zero_()
        v, rel = s.solve_v_cycle(rtol=1e-10, precision=prec)
        assert rel <= 1e-10
        r, nr = s.residual()
        assert nr / float(b.norm()) <= 1e-10 * (1 + 1e-6)
        res[fast] = (v, s.z.cpu().numpy().copy())
        print(kind, m, n, prec, "transform" if fast else "other", v)
    assert res[True][0] <= res[False][0]
    assert _rel(res[True][1], res[False][1]) < 1e-8


def test_transform_coarse_solve_not_used_where_it_does_not_apply(V):
    """The singular pure-Neumann MAC variant keeps its smoothed coarse path,
    the truncated viscous hierarchies have none."""
    neu = V.MgsMacNeumann(256, 128, 1 / 256, 1 / 256)
    assert neu.coarse_cycle()[1] != -1
    visc = V.ViscoImpl(256, 128, True, True, 5., 5.)
    assert visc.coarse_cycle() == (-1, 0)
