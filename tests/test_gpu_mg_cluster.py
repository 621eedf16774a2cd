"""The cluster-resident coarse cycle against the single-CTA coarse cycle.

MAC systems whose exact coarsest level has a finer neighbour that splits
into equal row slabs run their coarse levels in one thread-block-cluster
launch (VDI_MG_CLUSTER=0 restores the per-level tile kernels and the
single-CTA cycle). Both are the same V-cycle: red-black Gauss-Seidel(2,2),
averaging restriction, bilinear prolongation and the exact coarsest solve,
so iterates agree to rounding and solves take the same V-cycles."""
import numpy as np
import pytest

from test_gpu_mg import gaussians_rhs, _rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def V():
    import vdropimpact_b200 as V
    return V


# (m, n, first cluster level, CTAs): top levels 256x128 (2048x1024 down),
# 256x128 at level 1, the whole grid in the cluster, two slab levels of two
# rows and one row, and an 8-CTA cluster
CASES = [(2048, 1024, 3, 16), (512, 256, 1, 16), (256, 128, 0, 16), (64, 32, 0, 16), (96, 32, 0, 16),
         (2048, 128, 3, 8)]


def _system(V, m, n, cluster, monkeypatch):
    # the separable transform solve would take the coarse levels instead
    monkeypatch.setenv("VDI_MG_FAST_COARSE", "0")
    monkeypatch.setenv("VDI_MG_CLUSTER", "1" if cluster else "0")
    dx = 1.0 / m
    s = V.MgsMac(m, n, dx, 1.5 * dx)
    monkeypatch.delenv("VDI_MG_CLUSTER")
    monkeypatch.delenv("VDI_MG_FAST_COARSE")
    return s


@pytest.mark.parametrize("m,n,top,cs", CASES)
def test_cluster_vcycles_match_single_cta(V, m, n, top, cs, monkeypatch):
    import torch
    b = torch.from_numpy(gaussians_rhs(m, n, seed=11))
    out = {}
    for cluster in (True, False):
        s = _system(V, m, n, cluster, monkeypatch)
        first, ctas = s.coarse_cycle()
        if cluster:
            assert (first, ctas) == (top, cs)
        else:
            assert ctas == 1
        s.b.copy_(b)
        s.z.zero_()
        zs = []
        for _ in range(3):
            s.v_cycle()
            zs.append(s.z.cpu().numpy().copy())
        out[cluster] = zs
    for k in range(3):
        assert _rel(out[True][k], out[False][k]) < 1e-10, k


@pytest.mark.parametrize("prec", ["fp64", "mixed", "hybrid"])
@pytest.mark.parametrize("m,n,top,cs", CASES[:3] + CASES[5:])
def test_cluster_solves_match_single_cta(V, m, n, top, cs, prec, monkeypatch):
    import torch
    b = torch.from_numpy(gaussians_rhs(m, n, seed=5))
    res = {}
    for cluster in (True, False):
        s = _system(V, m, n, cluster, monkeypatch)
        s.b.copy_(b)
        s.z.zero_()
        v, rel = s.solve_v_cycle(rtol=1e-10, precision=prec)
        assert rel <= 1e-10
        r, nr = s.residual()
        assert nr / float(b.norm()) <= 1e-10 * (1 + 1e-6)
        res[cluster] = (v, s.z.cpu().numpy().copy())
    assert abs(res[True][0] - res[False][0]) <= 1
    assert _rel(res[True][1], res[False][1]) < 1e-8


def test_cluster_cycle_reports_single_cta_for_other_systems(V, monkeypatch):
    """The FEM, Neumann and viscous hierarchies keep their own coarse path:
    the FEM one solves its first CTA-sized level (65x33 here) exactly over
    the whole GPU (0 CTAs), or runs the single-CTA cycle with
    VDI_MG_FEM_DIRECT=0."""
    monkeypatch.setenv("VDI_MG_FAST_COARSE", "0")
    fem = V.MgsFem(129, 65, 1 / 128, 1 / 128)
    assert fem.coarse_cycle() == (1, 0)
    monkeypatch.setenv("VDI_MG_FEM_DIRECT", "0")
    fem = V.MgsFem(129, 65, 1 / 128, 1 / 128)
    monkeypatch.delenv("VDI_MG_FEM_DIRECT")
    monkeypatch.delenv("VDI_MG_FAST_COARSE")
    assert fem.coarse_cycle() == (1, 1)
    neu = V.MgsMacNeumann(256, 128, 1 / 256, 1 / 256)
    assert neu.coarse_cycle()[1] == 1
    visc = V.ViscoImpl(256, 128, True, True, 5., 5.)
    assert visc.coarse_cycle() == (-1, 0)


# FEM grids whose first CTA-sized level (65x33, 2145 nodes) is solved
# exactly over the whole GPU
FEM_CASES = [(2049, 1025, 5), (1025, 513, 4), (257, 129, 2)]


@pytest.mark.parametrize("prec", ["fp64", "mixed", "hybrid"])
@pytest.mark.parametrize("M,N,first", FEM_CASES)
def test_fem_direct_coarse_solve_matches_cta_cycle(V, M, N, first, prec, monkeypatch):
    """The whole-GPU exact solve of the coarse FEM level against the
    single-CTA cycle (smoothing down to the 256-node exact level): both
    solves reach the 1e-10 residual and agree to its accuracy; the exact
    coarse solve takes no more V-cycles."""
    import torch
    g = torch.Generator().manual_seed(M + N)
    b = torch.randn(M * N, dtype=torch.float64, generator=g)
    b[:M] = 0.3
    res = {}
    for direct in (True, False):
        monkeypatch.setenv("VDI_MG_FAST_COARSE", "0")
        monkeypatch.setenv("VDI_MG_FEM_DIRECT", "1" if direct else "0")
        s = V.MgsFem(M, N, 1.0 / (M - 1), 1.5 / (M - 1))
        monkeypatch.delenv("VDI_MG_FEM_DIRECT")
        monkeypatch.delenv("VDI_MG_FAST_COARSE")
        f, ctas = s.coarse_cycle(precision=prec if prec == "mixed" else None)
        if direct:
            assert (f, ctas) == (first, 0)
        else:
            assert ctas == 1
        s.b.copy_(b)
        s.z.zero_()
        v, rel = s.solve_v_cycle(rtol=1e-10, precision=prec)
        assert rel <= 1e-10
        r, nr = s.residual()
        assert nr / float(b.norm()) <= 1e-10 * (1 + 1e-6)
        res[direct] = (v, s.z.cpu().numpy().copy())
        print(M, N, prec, "direct" if direct else "cta", v)
    assert res[True][0] <= res[False][0]
    assert _rel(res[True][1], res[False][1]) < 1e-8
