"""Batched simulations (one CUDA graph per timestep, a branch per
simulation) and the autotuner: a batch steps each simulation exactly as it
steps alone, and tuning changes launch shapes and hierarchy cuts, not
results beyond the multigrid tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "p", "h", "pg", "gp", "tau", "fbd")


@pytest.fixture(scope="module")
def V():
    import vdropimpact_b200 as V
    return V


def test_batch_equals_individual_runs(V):
    cfgs = V.sweep_configs(6, seed=1, sizes=(64, 128, 256))
    b = V.Batch(cfgs)
    b.init_fields()
    dts = b.frame_dts()
    b.step_forward(dts, 20)
    for k, cfg in enumerate(cfgs):
        f = V.Fluid2D(cfg, graph=True)
        f.init_fields()
        f.step_forward(dts[k], 20)
        a, r = b.sims[k].state(), f.state()
        for name in FIELDS:
            assert np.array_equal(a[name], r[name]), (k, name)
        assert b.sims[k].stats()["steps"] == 20
        f.close()
    b.close()


def test_batch_reports_failing_simulation(V):
    cfgs = V.sweep_configs(3, seed=2, sizes=(64,))
    b = V.Batch(cfgs, mg_max_vcycles=1)
    b.init_fields()
    with pytest.raises(V.VdiError) as e:
        b.step_forward(b.frame_dts(), 2)
    assert "batch simulation 0" in str(e.value)
    b.close()


def test_autotune_keeps_results(V):
    cfg = V.sweep_configs(1, seed=3, sizes=(256,))[0]
    a = V.Fluid2D(cfg, graph=True)
    t = a.autotune()
    assert t["block"][0] * t["block"][1] <= 1024 and t["stencil_ms"] > 0
    assert all(x > 0 for x in t["vcycle_ms"][:2])
    b = V.Fluid2D(cfg, graph=True)
    t2 = b.autotune()
    assert t2["from_cache"] and t2["block"] == t["block"] and t2["cta_limit"] == t["cta_limit"]
    c = V.Fluid2D(cfg, graph=True)
    for f in (a, c):
        f.init_fields()
        f.step_forward(f.frame_dt(), 20)
    sa, sc = a.state(), c.state()
    for name in FIELDS:
        den = max(np.abs(sc[name]).max(), 1e-300)
        assert np.abs(sa[name] - sc[name]).max() / den < 1e-8, name


def test_batch_autotune(V):
    cfgs = V.sweep_configs(4, seed=4, sizes=(64, 128))
    b = V.Batch(cfgs)
    tunes = b.autotune()
    assert len(tunes) == 4
    sizes = [V.params_from_cfg(c).m for c in cfgs]
    for k in range(4):
        if sizes[k] in sizes[:k]:
            assert tunes[k]["from_cache"]
    b.init_fields()
    b.step_forward(b.frame_dts(), 10)
    assert all(s.stats()["steps"] == 10 for s in b.sims)
    b.close()
