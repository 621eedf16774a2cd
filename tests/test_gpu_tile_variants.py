"""The alternative kernels for the tiled multigrid levels (VDI_MG_TILE=reg,
reg1, tma) against the default shared-memory tiles: the same solves on the
same sources. The variants perform the same smoothing arithmetic on the
same points in the same order, so the V-cycle counts must be equal and the
FP64 solutions equal to the last bits. Their residual norms may differ in the
rounding noise that a converged residual consists of (the passes that
evaluate it order their sums differently), which could only change a count
at a threshold. Each variant runs in its own process, since the switch is read
once per process, and reports which path it took."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROG = r"""
import ctypes, json, sys
import torch
sys.path.insert(0, %r)
import vdropimpact_b200 as V
from vdropimpact_b200 import _abi
out = {}
for kind, m, n in (("mac", 1024, 512), ("mac", 600, 300), ("mac", 601, 300), ("fem", 1025, 513)):
    cls = V.MgsMac if kind == "mac" else V.MgsFem
    s = cls(m, n, 1. / m, 1.5 / m)
    g = torch.Generator(device="cuda").manual_seed(m + n)
    b = torch.randn(m * n, dtype=torch.float64, device="cuda", generator=g)
    if kind == "fem":
        b[:m] = 0.3
    s.b.copy_(b)
    r = {}
    for prec in ("fp64", "mixed"):
        s.z.zero_()
        v, rel = s.solve_v_cycle(1e-10, precision=None if prec == "fp64" else prec)
        r[prec] = dict(v=v, rel=rel, z=s.z[::997].cpu().tolist())
    out[f"{kind}{m}x{n}"] = r
    del s
pl = ctypes.c_longlong(0)
out["path"] = _abi.lib().vdi_mg_tile_path(ctypes.byref(pl))
out["persistent_launches"] = pl.value
print(json.dumps(out))
""" % ROOT


def run(variant):
    env = dict(os.environ)
    env.pop("VDI_MG_TILE", None)
    if variant:
        env["VDI_MG_TILE"] = variant
    r = subprocess.run([sys.executable, "-c", PROG], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.fixture(scope="module")
def default_run():
    return run(None)


@pytest.mark.parametrize("variant,path", [("reg", 1), ("reg1", 2), ("tma", 3)])
def test_tile_variant_matches_shared_memory_tiles(default_run, variant, path):
    base, alt = dict(default_run), run(variant)
    assert base.pop("path") == 0 and base.pop("persistent_launches") == 0
    assert alt.pop("path") == path
    launches = alt.pop("persistent_launches")
    # the persistent tile runs only where it applies: FP64 cell-centred levels
    assert (launches > 0) == (variant == "tma"), launches
    for key in base:
        for prec in ("fp64", "mixed"):
            x, y = base[key][prec], alt[key][prec]
            print(variant, key, prec, x["v"], y["v"], x["rel"], y["rel"])
            assert x["v"] == y["v"], (key, prec)
            # a converged residual is rounding noise of O(1) terms (about
            # 1e-16 of each against a residual near 1e-11 of ||b||): the
            # variants' own residual passes agree on it to about 1e-4
            assert y["rel"] <= 1e-10 and abs(x["rel"] - y["rel"]) <= 1e-3 * x["rel"]
            za, zb = np.array(x["z"]), np.array(y["z"])
            # FP64: the same arithmetic; the FP32 V-cycles of the mixed solve
            # may contract their FP32 sums into FMAs differently per kernel,
            # which moves the refined solution by rounding of that size
            tol = 1e-13 if prec == "fp64" else 1e-11
            assert np.abs(za - zb).max() <= tol * max(np.abs(za).max(), 1e-30), (key, prec)
