"""The learned initial guess where a guess can pay: the single-projection
workload solved from scratch. A U-Net trained on the GPU by this library's
own kernels, on (source, solution) pairs of seeded 64-Gaussian sources,
gives the initial guess of held-out solves (vdi_unet_guess). The test
asserts that it saves V-cycles against the zero guess, and that both solves
end at the same solution (each to ||b-Az|| <= 1e-10 ||b||, so within 1e-8 of
the solution's largest magnitude)."""
import pytest

pytestmark = pytest.mark.gpu


def test_learned_guess_saves_vcycles_on_fresh_solves():
    from vdropimpact_b200 import learned
    res = learned.config4_experiment(256, 128, 2, pairs=2000, iters=1500, batch=16, heldout=16)
    ev = res["eval"]["256x128"]
    print(res)
    assert res["loss_last"] < 0.2 * res["loss_first"], res
    assert ev["max_rel_diff_vs_zero_guess_solution"] < 1e-8, ev
    assert ev["vcycles_saved"] >= 1.0, ev
