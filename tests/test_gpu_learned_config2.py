"""The learned initial guess on the single-projection workload solved from
scratch (zero initial guess), where the network's prediction of the solution
is the whole guess. A U-Net trained on the GPU by this library's own kernels,
on (source, solution) pairs of seeded 64-Gaussian sources, gives the initial
guess of held-out solves through vdi_unet_guess.

What is asserted: training lowers the loss at least tenfold; the guess
captures the solution's large scales (its error, measured on 8 x 8 block
means, is well below that of the zero guess, which is 1); and the solve from
it ends at the same solution as the solve from zero (each to
||b-Az|| <= 1e-10 ||b||, so within 1e-8 of the solution's largest magnitude).
The V-cycle counts of both are printed. They are not asserted to favour the
network: a BF16 network's grid-scale error makes the starting residual of
its guess hundreds of times ||b||, and the V-cycles spend their reduction on
that before the better large scales show; at the contraction of these
V-cycles (about 0.06 to 0.1 with the exact transform solve of the 128 x 64
level) that costs up to three V-cycles more than the zero guess."""
import pytest

pytestmark = pytest.mark.gpu


def test_learned_guess_on_fresh_solves():
    from vdropimpact_b200 import learned
    res = learned.config4_experiment(256, 128, 2, pairs=2000, iters=1500, batch=16, heldout=16)
    ev = res["eval"]["256x128"]
    print(res)
    assert res["loss_last"] < 0.1 * res["loss_first"], res
    assert ev["guess_error_8x8_blocks"] < 0.5, ev
    assert ev["max_rel_diff_vs_zero_guess_solution"] < 1e-8, ev
    assert ev["vcycles_learned"] <= ev["vcycles_zero_guess"] + 3, ev
