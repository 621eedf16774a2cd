"""The viscous boundary kernel without barriers (many blocks, each column
recomputing what the single-CTA kernel's earlier phases leave in the cells
it reads, fluid_2d_sio.cc:294-343) against the single-CTA kernel
(VDI_VISC_BC_PAR=0): whole runs agree bit for bit, with and without the
x symmetry, in CUDA graphs and launched one by one."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("sym", [True, False])
@pytest.mark.parametrize("graph", [True, False])
def test_barrier_free_viscous_bc_same_bits(sym, graph, monkeypatch):
    import vdropimpact_b200 as V
    text = open(os.path.join(HERE, "golden", "ld_vis100.cfg")).read().replace("grid_points 2048 1024",
                                                                               "grid_points 256 128")
    if not sym:
        text = text.replace("\nx_sym\n", "\n")
    res = {}
    for par in ("1", "0"):
        monkeypatch.setenv("VDI_VISC_BC_PAR", par)
        f = V.Fluid2D(text, mg_rtol=1e-10, mg_guess="quadratic", graph=graph)
        f.init_fields()
        f.step_forward(f.frame_dt(), 12)
        res[par] = {k: np.asarray(v).copy() for k, v in f.state().items() if k not in ("m", "n")}
        f.close()
        monkeypatch.delenv("VDI_VISC_BC_PAR")
    for k in res["0"]:
        assert np.array_equal(res["1"][k], res["0"][k]), k


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("graph", [True, False])
def test_viscous_guesses_beside_mac_solve_same_bits(prec, graph, monkeypatch):
    """The two viscous guesses run on the side stream beside the MAC solve,
    extrapolating to the time the MAC correction sets (the clock the gas
    layer left plus dt/2, the same sum the correction forms); whole runs
    equal those with the guesses on the viscous solves' own streams
    (VDI_VISC_GUESS_SIDE=0) bit for bit."""
    import vdropimpact_b200 as V
    text = open(os.path.join(HERE, "golden", "ld_vis100.cfg")).read().replace("grid_points 2048 1024",
                                                                               "grid_points 256 128")
    res = {}
    for side in ("1", "0"):
        monkeypatch.setenv("VDI_VISC_GUESS_SIDE", side)
        f = V.Fluid2D(text, mg_rtol=1e-10, mg_precision=prec, mg_guess="quadratic", graph=graph)
        monkeypatch.delenv("VDI_VISC_GUESS_SIDE")
        f.init_fields()
        f.step_forward(f.frame_dt(), 12)
        st = f.stats()
        res[side] = ({k: np.asarray(v).copy() for k, v in f.state().items() if k not in ("m", "n")},
                     st["vcycles"])
        f.close()
    assert res["1"][1] == res["0"][1]
    for k in res["0"][0]:
        assert np.array_equal(res["1"][0][k], res["0"][0][k]), k
