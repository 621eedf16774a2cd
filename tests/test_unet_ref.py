"""Pins the CPU float64 U-Net reference (tests/unet_ref.py) used by the GPU
numerics tests: its autograd weight gradients against central finite
differences of its own float64 forward, and its layer table against the
network description (14 layers, 221,712 parameters)."""
import numpy as np

import unet_ref


def _params(seed):
    g = np.random.default_rng(seed)
    out = []
    for ci, co, *_ in unet_ref.SPEC:
        out.append(((g.uniform(-1, 1, (9, co, ci)) * np.sqrt(6 / (9 * ci))),
                    0.01 * g.standard_normal(co)))
    return out


def test_layer_table():
    assert len(unet_ref.SPEC) == 14
    assert unet_ref.param_count() == 221_712
    flat = np.arange(unet_ref.param_count(), dtype=np.float32)
    parts = unet_ref.split_params(flat)
    assert parts[0][0].shape == (9, 16, 16) and parts[4][0].shape == (9, 64, 32)
    assert parts[-1][1][-1] == flat[-1]


def test_gradients_match_finite_differences():
    prm = _params(0)
    g = np.random.default_rng(1)
    x = g.standard_normal((1, 16, 32))
    t = 0.3 * g.standard_normal((1, 16, 32))
    _, grads = unet_ref.loss_and_grads(prm, x, t, bf16=False)
    import torch
    eps = 1e-6
    for k, (tap, co, ci) in [(0, (4, 3, 0)), (4, (1, 7, 5)), (8, (8, 2, 60)), (13, (4, 0, 3))]:
        vals = []
        for s in (1, -1):
            p2 = [(w.copy(), b) for w, b in prm]
            p2[k][0][tap, co, ci] += s * eps
            y, _ = unet_ref.forward(p2, x, bf16=False)
            vals.append(float(torch.mean((y - torch.as_tensor(t)) ** 2)))
        fd = (vals[0] - vals[1]) / (2 * eps)
        assert abs(fd - grads[k][tap, co, ci]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, grads[k][tap, co, ci])
