"""The U-Net's convolutions on the Blackwell tensor cores (tcgen05.mma with
TMEM accumulators, VDI_UNET_TC=1) against the mma.sync kernels: forward
outputs and weight gradients of the same network on the same inputs.
Both use BF16 operands and FP32 accumulation, and only the order of the FP32
sums differs; but each layer stores its output in BF16, so a sum that lands
near a rounding boundary can round the other way (a relative step of 2^-8)
and carry that into the next layers. The tolerance, 5e-3 of each quantity's
largest magnitude, is that BF16 step with a margin. Each configuration runs
in its own process, since the switch is read once per process."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROG = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, %r)
from vdropimpact_b200 import learned, _abi
out = {"path": _abi.lib().vdi_unet_tensor_path()}
for (H, W) in ((32, 128), (24, 48), (64, 256)):
    net = learned.UNet(H, W, batch=2, seed=5)
    g = torch.Generator(device="cuda").manual_seed(H + W)
    x = torch.randn(2, H, W, device="cuda", generator=g, dtype=torch.float32)
    t = torch.randn(2, H, W, device="cuda", generator=g, dtype=torch.float32)
    y = net.forward(x)
    gr, loss = net.gradients(x, t, 4, (9, 64, 32))
    g0, _ = net.gradients(x, t, 0, (9, 16, 16))
    out[f"{H}x{W}"] = dict(y=y.cpu().numpy().ravel().tolist(), g4=gr.ravel().tolist(), g0=g0.ravel().tolist(),
                          loss=loss)
print(json.dumps(out))
""" % ROOT


def run(tc: bool):
    env = dict(os.environ, VDI_UNET_TC="1" if tc else "0")
    r = subprocess.run([sys.executable, "-c", PROG], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_tensor_core_convolutions_match_mma_sync():
    a, b = run(False), run(True)
    assert a.pop("path") == 0 and b.pop("path") == 1
    for key in a:
        for f in ("y", "g4", "g0"):
            x, y = np.array(a[key][f]), np.array(b[key][f])
            scale = max(np.abs(x).max(), 1e-30)
            err = np.abs(x - y).max() / scale
            print(key, f, err)
            assert err < 5e-3, (key, f, err)
        assert abs(a[key]["loss"] - b[key]["loss"]) <= 5e-3 * abs(a[key]["loss"]), key
