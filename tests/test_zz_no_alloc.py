"""The allocation-free multigrid solve (vdi_mg_solve_noalloc) against the
allocating one (vdi_mg_create + vdi_mg_solve), called through the C ABI.

The allocation-free entry point serves callers that cannot allocate device
memory (an application that owns every allocation, or code where an
allocation would stall); it takes its scratch from one static device array.
Each case makes two calls in a row, since the array keeps the previous
call's contents."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _gauss(m, n, seed):
    rng = np.random.default_rng(seed)
    x = (np.arange(m) + 0.5) / m
    y = (np.arange(n) + 0.5) / m
    X, Y = np.meshgrid(x, y)
    b = np.zeros((n, m))
    for _ in range(16):
        cx, cy, w = rng.uniform(0, 1), rng.uniform(0, n / m), rng.uniform(0.02, 0.1)
        b += rng.standard_normal() * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * w * w))
    return (b - b.mean()).ravel()


def _solve_allocating(L, kind, m, n, c1, c2, x_sym, b):
    import torch
    from vdropimpact_b200 import _abi
    h = C.c_void_p()
    _abi.check(L.vdi_mg_create(kind, m, n, c1, c2, x_sym, None, C.byref(h)), "vdi_mg_create")
    db = torch.from_numpy(b).cuda()
    dz = torch.zeros_like(db)
    r = _abi.VdiMgResult()
    torch.cuda.synchronize()
    _abi.check(L.vdi_mg_solve(h, C.c_void_p(db.data_ptr()), C.c_void_p(dz.data_ptr()), 1e-10, 200, 0,
                              C.byref(r)), "vdi_mg_solve")
    L.vdi_mg_destroy(h)
    return dz.cpu().numpy(), r.vcycles


def _solve_noalloc(L, kind, m, n, c1, c2, x_sym, b):
    import torch
    from vdropimpact_b200 import _abi
    db = torch.from_numpy(b).cuda()
    dz = torch.zeros_like(db)
    r = _abi.VdiMgResult()
    torch.cuda.synchronize()
    st = L.vdi_mg_solve_noalloc(kind, m, n, C.c_double(c1), C.c_double(c2), x_sym, C.c_void_p(db.data_ptr()),
                                C.c_void_p(dz.data_ptr()), C.c_double(1e-10), 200, None, C.byref(r))
    _abi.check(st, "vdi_mg_solve_noalloc")
    return dz.cpu().numpy(), r.vcycles


@pytest.fixture(scope="module")
def L():
    from vdropimpact_b200 import _abi
    lib = _abi.lib()
    f = lib.vdi_mg_solve_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_void_p,
                  C.c_double, C.c_int, C.c_void_p, C.POINTER(_abi.VdiMgResult)]
    return lib


@pytest.mark.parametrize("kind,m,n,c1,c2,x_sym", [
    (0, 256, 128, 1. / 256, 1. / 256, 0),      # MAC, dx, dy
    (1, 257, 129, 1. / 256, 1. / 256, 0),      # FEM nodes, dx, dy
    (2, 256, 128, 0.4, 0.4, 1),                # viscous u, vfx, vfy
])
def test_noalloc_matches_allocating_solve_twice(L, kind, m, n, c1, c2, x_sym):
    for call, seed in enumerate((3, 4)):
        b = _gauss(m, n, seed)
        if kind == 1:
            b = b.reshape(n, m)
            b[0, :] = 50.0
            b = b.ravel()
        za, va = _solve_allocating(L, kind, m, n, c1, c2, x_sym, b)
        zn, vn = _solve_noalloc(L, kind, m, n, c1, c2, x_sym, b)
        scale = max(np.abs(za).max(), 1e-300)
        assert np.abs(zn - za).max() / scale <= TOL, (kind, call)
        assert vn == va, (kind, call)


def test_noalloc_rejects_oversized_grid(L):
    import torch
    from vdropimpact_b200 import _abi
    m, n = 1024, 512
    db = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    dz = torch.zeros_like(db)
    r = _abi.VdiMgResult()
    st = L.vdi_mg_solve_noalloc(0, m, n, C.c_double(1. / m), C.c_double(1. / m), 0, C.c_void_p(db.data_ptr()),
                                C.c_void_p(dz.data_ptr()), C.c_double(1e-10), 200, None, C.byref(r))
    assert st == _abi.VDI_ERR_UNSUPPORTED_SIZE
    assert b"exceeds the maximum" in L.vdi_last_error()
