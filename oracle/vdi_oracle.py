"""ORACLE TEST INFRASTRUCTURE — not part of the product.

A CPU restatement, in numpy, of vdropimpact's per-timestep fluid solve. Only
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
use it, and only as the checker. Each function cites the reference lines it
restates (paths relative to the vdropimpact repository).

Arrays use the reference's ghosted layout: a field over the liquid grid has
shape (n+4, m+4), and cell (i, j) sits at [j+2, i+2]. Pressure lives at grid
nodes (i <= m, j <= n) in the same array (fluid_2d.cc:383-396). Expressions
keep the reference's evaluation order, so the stencil work matches the
reference bit for bit when both run without FMA contraction.

The linear systems are solved exactly with a sparse LU factorisation. That is
the limit that the reference's multigrid V-cycles converge to, not the
V-cycles themselves: TGMG (the reference's multigrid engine) is not
available, and its V-cycle counts are not part of the restatement.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

EPS = np.finfo(np.float64).eps
# gas_layer_solve.hh:11-18
PRESSURE_R_ERROR = EPS * 1e8
NEWTON_THRESH = PRESSURE_R_ERROR * PRESSURE_R_ERROR
MAX_NEWTON_STEPS = 256


class OracleError(RuntimeError):
    """Raised where the reference would call fatal_error() and exit."""


# --------------------------------------------------------------------------
# Configuration (fileinfo.cc:11-193, fluid_2d.cc:14-24, fluid_2d.hh:82-86)
# --------------------------------------------------------------------------
@dataclass
class Params:
    m: int
    n: int
    L_nd: float
    h0_nd: float
    t_end_nd: float
    nframes: int
    tmult: float
    nul: float
    rho: float
    R: float
    V: float
    alpha: float
    sigma: float
    mug: float
    Pamb: float
    x_sym: bool = False
    implicit_visc: bool = False
    # tracers and the non-inertial frame (fileinfo.cc:59, 96-101)
    ntrace: int = 0
    nif_mode: int = 0
    nif_r: float = 0.
    # derived
    mu: float = field(init=False)
    muinv: float = field(init=False)
    rhoinv: float = field(init=False)
    L: float = field(init=False)
    h0: float = field(init=False)
    t_end: float = field(init=False)
    ax: float = field(init=False)
    ay: float = field(init=False)
    bx: float = field(init=False)
    by: float = field(init=False)
    dx: float = field(init=False)
    dy: float = field(init=False)
    xsp: float = field(init=False)
    ysp: float = field(init=False)
    xxsp: float = field(init=False)
    yysp: float = field(init=False)
    dt_reg: float = field(init=False)
    nif_a: int = field(init=False)
    nif_b: int = field(init=False)

    def __post_init__(self):
        # fileinfo.cc:142-152
        self.mu = self.nul * self.rho
        self.muinv = 1. / self.mu
        self.rhoinv = 1. / self.rho
        st = self.mug / (self.rho * self.V * self.R)
        st3 = math.pow(st, 1. / 3.)
        st23 = st3 * st3
        self.L = self.L_nd * self.R * st3
        self.h0 = self.h0_nd * self.R * st23
        self.t_end = self.t_end_nd * self.R * st23 / self.V
        self.bx = self.L
        self.by = self.L * self.n / self.m
        self.ay = 0.
        if self.x_sym:
            self.ax = 0.
        else:
            self.ax = -self.L
            self.by *= 2
        # fluid_2d.cc:15-17
        self.dx = (self.bx - self.ax) / self.m
        self.dy = (self.by - self.ay) / self.n
        self.xsp = 1. / self.dx
        self.ysp = 1. / self.dy
        self.xxsp = self.xsp * self.xsp
        self.yysp = self.ysp * self.ysp
        if self.implicit_visc:
            self.dt_reg = self.dx * self.tmult
        else:
            self.dt_reg = self.dx * self.dx * self.rho * self.muinv * self.tmult * 0.25
        # fileinfo.cc:179-191: the nif_range window of columns
        self.nif_a = self.nif_b = 0
        if self.nif_mode == 2:
            b = int((self.nif_r - self.ax) * self.xsp + 0.5)
            if b >= self.m:
                b = self.m - 1
            if self.x_sym:
                a = 0
            else:
                a = max(0, int((-self.nif_r - self.ax) * self.xsp + 0.5))
            if b - a <= 0:
                raise OracleError("Velocity window for non-inertial frame is too small")
            self.nif_a, self.nif_b = a, b

    def timestep_select(self, interval: float):
        """fluid_2d.hh:82-86: largest dt <= dt_reg that divides interval."""
        l = int(interval / self.dt_reg) + 1
        return l, interval / l

    def frame_dt(self) -> float:
        """The timestep fluid_2d::solve uses (fluid_2d.cc:42)."""
        return self.timestep_select(self.t_end / self.nframes)[1]


def parse_cfg(text: str, **overrides) -> Params:
    """Keyword parser for the subset of fileinfo.cc:35-126 that the solve
    path needs (gas_layer_model only; tracers and output flags are read and
    ignored because they do not affect the fields)."""
    kv = {}
    flags = set()
    for raw in text.splitlines():
        line = raw.split('#', 1)[0].split()
        if not line:
            continue
        key, vals = line[0], line[1:]
        if key == 'grid_points':
            kv['m'], kv['n'] = int(vals[0]), int(vals[1])
        elif key in ('L_nd', 'h0_nd', 't_end_nd', 'tmult', 'R', 'V', 'sigma', 'mug', 'Pamb'):
            kv[key] = float(vals[0])
        elif key == 'frames':
            kv['nframes'] = int(vals[0])
        elif key == 'nul':
            kv['nul'] = float(vals[0])
        elif key == 'nul_cSt':
            kv['nul'] = 1e-6 * float(vals[0])
        elif key == 'rhol':
            kv['rho'] = float(vals[0])
        elif key == 'gamma':
            kv['alpha'] = 1. / float(vals[0])
        elif key == 'alpha':
            kv['alpha'] = float(vals[0])
        elif key in ('x_sym', 'implicit_visc', 'gas_layer_model', 'mr_time_output'):
            flags.add(key)
        elif key == 'tracers':
            kv['ntrace'] = int(vals[0])
        elif key == 'nif_center':
            kv['nif_mode'] = 1
        elif key == 'nif_range':
            kv['nif_mode'], kv['nif_r'] = 2, float(vals[0])
        elif key in ('restart_freq', 'output', 'gas_layer_data'):
            if key == 'gas_layer_data':
                raise OracleError(f"option {key} is outside the restated path")
        else:
            raise OracleError(f"Keyword '{key}' not understood")
    if 'gas_layer_model' not in flags:
        raise OracleError("gas_layer_model must be set")
    kv.update(overrides)
    return Params(x_sym='x_sym' in flags, implicit_visc='implicit_visc' in flags, **kv)


# --------------------------------------------------------------------------
# Linear systems (mgs_mac.hh:25-50, mgs_fem.hh:42-57 + mgs_fem.cc:8-53,
# visco_impl.hh:28-53), assembled from the stencil accessors.
# --------------------------------------------------------------------------
def _assemble(m, n, diag, left, right, down, up, dl=None, dr=None, ul=None, ur=None):
    """Builds a CSR matrix from per-point stencil arrays of shape (n, m)."""
    idx = np.arange(m * n).reshape(n, m)
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [diag.ravel()]

    def add(coef, di, dj):
        if coef is None:
            return
        c = np.asarray(coef, dtype=np.float64)
        j0, j1 = max(0, -dj), n - max(0, dj)
        i0, i1 = max(0, -di), m - max(0, di)
        cc = c[j0:j1, i0:i1]
        r = idx[j0:j1, i0:i1]
        g = idx[j0 + dj:j1 + dj, i0 + di:i1 + di]
        mask = cc != 0
        rows.append(r[mask]); cols.append(g[mask]); vals.append(cc[mask])

    add(left, -1, 0); add(right, 1, 0); add(down, 0, -1); add(up, 0, 1)
    add(dl, -1, -1); add(dr, 1, -1); add(ul, -1, 1); add(ur, 1, 1)
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(m * n, m * n))


def mac_matrix(m, n, xxsp, yysp, neumann_bottom=False):
    """mgs_mac.hh:33-48: cell-centred 5-point Laplacian, Neumann on the left,
    right and top, Dirichlet (ghost reflection, -3*yysp) on the bottom; with
    neumann_bottom the bottom is Neumann too (the pure-Neumann variant, which
    the reference does not have)."""
    i = np.arange(m)[None, :].repeat(n, 0)
    j = np.arange(n)[:, None].repeat(m, 1)
    diag = np.where((i > 0) & (i < m - 1), -2 * xxsp, -xxsp) + \
        np.where(j == 0, (-1 if neumann_bottom else -3) * yysp, np.where(j < n - 1, -2 * yysp, -yysp))
    left = np.where(i > 0, xxsp, 0.); right = np.where(i < m - 1, xxsp, 0.)
    down = np.where(j > 0, yysp, 0.); up = np.where(j < n - 1, yysp, 0.)
    return _assemble(m, n, diag, left, right, down, up)


def mac_direct_solve(m, n, xxsp, yysp, b):
    """Exact solve of mac_matrix(m, n, xxsp, yysp) z = b (mgs_mac.hh:33-48)
    for large grids, by separation of variables. The operator is
    T_x (x) I + I (x) T_y with T_x the cell-centred Neumann-Neumann second
    difference, which the orthonormal DCT-II diagonalises (eigenvalues
    -4 xxsp sin^2(pi k / 2m)), and T_y tridiagonal (Dirichlet ghost reflection
    at the bottom, Neumann at the top). So: DCT-II along x, one tridiagonal
    solve in y per mode (the Thomas algorithm, vectorised over the modes;
    every system is symmetric negative definite), inverse DCT. Cost
    O(m n log m); accuracy that of FP64 arithmetic on the conditioning of the
    system, with no iteration to converge."""
    import scipy.fft as sfft
    B = np.asarray(b, dtype=np.float64).reshape(n, m)
    Bh = sfft.dct(B, type=2, norm="ortho", axis=1)
    mu = -4. * xxsp * np.sin(np.pi * np.arange(m) / (2. * m)) ** 2
    d = np.empty((n, m))
    d[:] = -2. * yysp
    d[0] = -3. * yysp
    d[n - 1] = -yysp if n > 1 else -3. * yysp
    d += mu[None, :]
    c = np.empty((n, m))
    y = np.empty((n, m))
    c[0] = yysp / d[0]
    y[0] = Bh[0] / d[0]
    for j in range(1, n):
        den = d[j] - yysp * c[j - 1]
        c[j] = yysp / den
        y[j] = (Bh[j] - yysp * y[j - 1]) / den
    Z = np.empty((n, m))
    Z[n - 1] = y[n - 1]
    for j in range(n - 2, -1, -1):
        Z[j] = y[j] - c[j] * Z[j + 1]
    return sfft.idct(Z, type=2, norm="ortho", axis=1).ravel()


def fem_coeffs(dx, dy):
    """mgs_fem.cc:8-11: the bilinear finite-element stencil constants."""
    dydx, dxdy = dy / dx, dx / dy
    fm = 4. / 3. * (dxdy + dydx)
    fey = 1. / 3. * (-2 * dxdy + dydx)
    fex = 1. / 3. * (-2 * dydx + dxdy)
    fc = -1. / 6. * (dxdy + dydx)
    return dict(fm=fm, fey=fey, hey=0.5 * fey, fex=fex, hex=0.5 * fex, fc=fc)


def fem_a_cc(M, N, i, j, fm):
    """mgs_fem.hh:55-57."""
    return np.where((i > 0) & (i < M - 1), 1., 0.5) * np.where((j >= 1) & (j < N - 1), 1., 0.5) * fm


def fem_matrix(M, N, dx, dy):
    """mgs_fem.hh:42-57 and mgs_fem.cc:32-53 on an M x N node grid: 9-point
    stencil with half weights on the side and top edges; the bottom row is a
    Dirichlet row (only the diagonal)."""
    c = fem_coeffs(dx, dy)
    i = np.arange(M)[None, :].repeat(N, 0)
    j = np.arange(N)[:, None].repeat(M, 1)
    nb = j > 0
    inter_i = (i > 0) & (i < M - 1)
    mid_j = (j >= 1) & (j < N - 1)
    diag = fem_a_cc(M, N, i, j, c['fm'])
    dl = np.where(nb & (i > 0), c['fc'], 0.)
    dr = np.where(nb & (i < M - 1), c['fc'], 0.)
    ul = np.where(nb & (j < N - 1) & (i > 0), c['fc'], 0.)
    ur = np.where(nb & (j < N - 1) & (i < M - 1), c['fc'], 0.)
    down = np.where(nb, np.where(inter_i, c['fey'], c['hey']), 0.)
    up = np.where(nb & (j < N - 1), np.where(inter_i, c['fey'], c['hey']), 0.)
    left = np.where(nb & (i > 0), np.where(mid_j, c['fex'], c['hex']), 0.)
    right = np.where(nb & (i < M - 1), np.where(mid_j, c['fex'], c['hex']), 0.)
    return _assemble(M, N, diag, left, right, down, up, dl, dr, ul, ur)


def visco_matrix(m, n, vfx, vfy, x_sym, horizontal):
    """visco_impl.hh:28-53: (I - vfx Dxx - vfy Dyy) with a Neumann bottom,
    Dirichlet right/top (folded into the source), and at x=0 either the
    antisymmetric (u, 3*vfx) or symmetric (v, vfx) reflection when x_sym."""
    i = np.arange(m)[None, :].repeat(n, 0)
    j = np.arange(n)[:, None].repeat(m, 1)
    if x_sym:
        diag = 1 + np.where(i > 0, 2 * vfx, 3 * vfx if horizontal else vfx) + np.where(j > 0, 2 * vfy, vfy)
    else:
        diag = 1 + 2 * vfx + np.where(j > 0, 2 * vfy, vfy)
    left = np.where(i > 0, -vfx, 0.); right = np.where(i < m - 1, -vfx, 0.)
    down = np.where(j > 0, -vfy, 0.); up = np.where(j < n - 1, -vfy, 0.)
    return _assemble(m, n, diag, left, right, down, up)


class DirectSolver:
    """Exact solve of one of the systems (sparse LU, factored once)."""

    def __init__(self, A):
        self.A = A.tocsc()
        self.lu = spla.splu(self.A)

    def solve(self, b):
        return self.lu.solve(np.ascontiguousarray(b, dtype=np.float64))


# --------------------------------------------------------------------------
# Tridiagonal solve (tri_solve.cc:24-49)
# --------------------------------------------------------------------------
def dgtsv(dl, d, du, b):
    """Gaussian elimination with partial pivoting for a tridiagonal system,
    the algorithm of LAPACK's dgtsv that tri_solve::solve_lapack calls
    (tri_solve.cc:24-33). dl: n-1 sub-diagonal, d: n diagonal, du: n-1
    super-diagonal, b: right-hand side. Returns (x, info) like LAPACK."""
    n = len(d)
    dl = np.array(dl, dtype=np.float64); d = np.array(d, dtype=np.float64)
    du = np.array(du, dtype=np.float64); b = np.array(b, dtype=np.float64)
    du2 = np.zeros(max(n - 2, 0))
    for i in range(n - 1):
        if abs(d[i]) >= abs(dl[i]):
            if d[i] == 0:
                return b, i + 1
            fact = dl[i] / d[i]
            d[i + 1] -= fact * du[i]
            b[i + 1] -= fact * b[i]
            if i < n - 2:
                du2[i] = 0.
        else:
            fact = d[i] / dl[i]
            d[i] = dl[i]
            temp = d[i + 1]
            d[i + 1] = du[i] - fact * temp
            if i < n - 2:
                du2[i] = du[i + 1]
                du[i + 1] = -fact * du2[i]
            du[i] = temp
            temp = b[i]
            b[i] = b[i + 1]
            b[i + 1] = temp - fact * b[i + 1]
    if d[n - 1] == 0:
        return b, n
    b[n - 1] /= d[n - 1]
    if n > 1:
        b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2]
    for i in range(n - 3, -1, -1):
        b[i] = (b[i] - du[i] * b[i + 1] - du2[i] * b[i + 2]) / d[i]
    return b, 0


def thomas(a, b, c, d):
    """tri_solve::solve (tri_solve.cc:37-49): a[i] sub-diagonal of row i,
    c[i] super-diagonal of row i. Returns the solution."""
    a = np.array(a, float); b = np.array(b, float); c = np.array(c, float); d = np.array(d, float)
    m = len(b)
    c[0] /= b[0]
    for i in range(1, m - 1):
        c[i] /= b[i] - a[i] * c[i - 1]
    d[0] /= b[0]
    for i in range(1, m):
        d[i] = (d[i] - a[i] * d[i - 1]) / (b[i] - a[i] * c[i - 1])
    for i in range(m - 2, -1, -1):
        d[i] -= c[i] * d[i + 1]
    return d


# --------------------------------------------------------------------------
# Godunov helpers (fluid_2d.cc:419-476)
# --------------------------------------------------------------------------
def delta_lim(f0, f1, f2):
    """fluid_2d.cc:445-449."""
    drm = f1 - f0
    drp = f2 - f1
    return np.where(drm > 0, np.where(drp > 0, 2 * np.minimum(drm, drp), 0.),
                    np.where(drp > 0, 0., -2 * np.maximum(drm, drp)))


def delta_f(f0, f1, f2):
    """fluid_2d.cc:434-437."""
    drc = 0.5 * (f2 - f0)
    dl = delta_lim(f0, f1, f2)
    return np.where(drc > 0, np.minimum(drc, dl), np.maximum(drc, -dl))


def mono_diff(f0, f1, f2, f3, f4):
    """fluid_2d.cc:422-426: fourth-order monotonicity-limited slope."""
    tdrc = f3 - f1
    s = (1 / 6.) * (4 * tdrc - delta_f(f0, f1, f2) - delta_f(f2, f3, f4))
    t = delta_lim(f1, f2, f3)
    return np.where(tdrc > 0, np.minimum(s, t), np.maximum(s, -t))


def _min(a, b):
    # fluid_2d.hh:123: a<b?a:b (np.minimum differs only for NaN)
    return np.where(a < b, a, b)


def godunov_set_tang(u0, u1, v0, v1):
    """fluid_2d.cc:469-476. Returns the new (u0, u1, v1)."""
    c1 = u0 > -u1
    A = c1 & (u0 > 0)
    B = (~c1) & (u1 < 0)
    C = ~(A | B)
    nu0 = np.where(B, u1, np.where(C, 0.5 * (u0 + u1), u0))
    nu1 = np.where(A, u0, np.where(C, 0., u1))
    nv1 = np.where(A, v0, np.where(C, 0.5 * (v0 + v1), v1))
    return nu0, nu1, nv1


def godunov_set(u0, u1, v0, v1):
    """fluid_2d.cc:455-461. Returns the new (u1, v1)."""
    c1 = u0 > -u1
    A = c1 & (u0 > 0)
    B = (~c1) & (u1 < 0)
    C = ~(A | B)
    nu1 = np.where(A, u0, np.where(C, 0., u1))
    nv1 = np.where(A, v0, np.where(C, 0.5 * (v0 + v1), v1))
    return nu1, nv1


# --------------------------------------------------------------------------
# The simulation
# --------------------------------------------------------------------------
class Oracle:
    """State and step of fluid_2d + gas_layer_solve (x_sym or not,
    implicit or explicit viscosity, gas_layer_model, tracers, inertial or
    non-inertial frame)."""

    def __init__(self, prm: Params):
        self.prm = prm
        m, n = prm.m, prm.n
        self.m, self.n, self.me, self.ne, self.ml = m, n, m + 1, n + 1, m + 4
        shp = (n + 4, m + 4)
        self.u = np.zeros(shp); self.v = np.zeros(shp); self.p = np.zeros(shp)
        self.time = 0.
        # gas layer (gas_layer.cc:8-13, gas_layer_solve.cc:8-15)
        self.Vframe = prm.V
        self.gp = np.zeros(m + 1)      # gas_layer::p (liquid pressure at the base)
        self.tau = np.zeros(m + 4)
        self.gp_old = np.zeros(m + 1)
        self.tau_old = np.zeros(m + 4)
        self.h = np.zeros(m); self.hx = np.zeros(m + 1); self.ht = np.zeros(m)
        self.fbd = np.zeros(m); self.pg = np.zeros(m + 1); self.pg_old = np.zeros(m + 1)
        self._solvers = {}
        self.newton_iters = []
        self.tm = np.zeros(2 * prm.ntrace)   # tracer positions x0, y0, x1, ...

    # -------------------------------------------------- index helpers
    def S(self, a, di=0, dj=0):
        """View of a over the m x n cells shifted by (di, dj)."""
        m, n = self.m, self.n
        return a[2 + dj:2 + dj + n, 2 + di:2 + di + m]

    def N(self, a, di=0, dj=0):
        """View of a over the (m+1) x (n+1) nodes shifted by (di, dj)."""
        m, n = self.m, self.n
        return a[2 + dj:3 + dj + n, 2 + di:3 + di + m]

    # -------------------------------------------------- initialisation
    def init_fields(self):
        """fluid_2d_sio.cc:14-35 and gas_layer_solve.cc:32-53."""
        prm = self.prm
        self.time = 0.
        self.u[:] = 0; self.v[:] = 0; self.p[:] = 0
        m = self.m
        self.fbd[:] = 0
        x = prm.ax + (np.arange(m) + 0.5) * prm.dx
        self.h[:] = prm.h0 + 0.5 / prm.R * x * x
        self.calculate_hx()
        self.ht[:] = -prm.V
        self.pg[:] = 0
        self.calculate_liquid_fields()
        self.set_boundaries(0.)
        if prm.ntrace > 0:
            self.init_tracers()

    def init_tracers(self):
        """fluid_2d::init_tracers (fluid_2d.cc:495-502) with the C library's
        rand() of this process (the reference's positions in a process that
        has not called rand() before)."""
        import ctypes
        import ctypes.util
        libc = ctypes.CDLL(ctypes.util.find_library("c"))
        rand_max = 2147483647     # glibc RAND_MAX
        prm = self.prm
        for k in range(0, self.tm.size, 2):
            self.tm[k] = prm.ax + (prm.bx - prm.ax) / rand_max * float(libc.rand())
            self.tm[k + 1] = prm.ay + (prm.by - prm.ay) / rand_max * float(libc.rand())

    def update_tracers(self, dt):
        """fluid_2d::update_tracers (fluid_2d.cc:507-526): bilinear
        interpolation of the cell-centred velocity, cell index clamped to
        [-1, m-1] x [-1, n-1]."""
        if self.tm.size == 0:
            return
        prm = self.prm
        x = (self.tm[0::2] - prm.ax) * prm.xsp - 0.5
        y = (self.tm[1::2] - prm.ay) * prm.ysp - 0.5
        i = np.clip(np.trunc(x).astype(np.int64), -1, self.m - 1)
        j = np.clip(np.trunc(y).astype(np.int64), -1, self.n - 1)
        x = x - i
        y = y - j
        r, c = j + 2, i + 2
        for k, f in ((0, self.u), (1, self.v)):
            val = (1 - y) * (f[r, c] * (1 - x) + f[r, c + 1] * x) + y * (f[r + 1, c] * (1 - x) + f[r + 1, c + 1] * x)
            self.tm[k::2] += dt * val

    def adjust_frame(self):
        """fluid_2d::adjust_frame (fluid_2d_sio.cc:228-253)."""
        prm, m = self.prm, self.m
        fm = self.v[2, 2:]      # row 0
        fb = self.v[1, 2:]      # row -1
        if prm.nif_mode == 1:
            m2 = m // 2
            if prm.x_sym:
                V = 0.5625 * (fb[0] + fm[0]) - 0.0625 * (fb[1] + fm[1])
            else:
                V = (0.28125 * (fb[m2 - 1] + fb[m2] + fm[m2 - 1] + fm[m2])
                     - 0.03125 * (fb[m2 - 2] + fb[m2 + 1] + fm[m2 - 2] + fm[m2 + 1]))
        else:
            V = 0.
            for i in range(prm.nif_a, prm.nif_b):
                V += float(fm[i]) + float(fb[i])
            V *= 0.5 / (prm.nif_b - prm.nif_a)
        self.v -= V
        self.Vframe -= V

    # -------------------------------------------------- gas layer
    def calculate_hx(self):
        """gas_layer_solve.cc:55-59."""
        m, xsp = self.m, self.prm.xsp
        self.hx[1:m] = xsp * (self.h[1:m] - self.h[0:m - 1])
        self.hx[0] = 0. if self.prm.x_sym else self.hx[1]
        self.hx[m] = self.hx[m - 1]

    def h_ref(self, i):
        """gas_layer_solve.cc:173-177."""
        h, m = self.h, self.m
        if i >= 0:
            return h[i] if i < m else (2 * h[m - 1] - h[m - 2] if i == m else 3 * h[m - 1] - 2 * h[m - 2])
        if self.prm.x_sym:
            return h[0] if i == -1 else h[1]
        return 2 * h[0] - h[1] if i == -1 else 3 * h[0] - 2 * h[1]

    @staticmethod
    def eno2(p0, p1, p2, p3):
        """gas_layer_solve.cc:165-167."""
        return 3 * p1 - 4 * p2 + p3 if abs(p0 - 2 * p1 + p2) > abs(p1 - 2 * p2 + p3) else p0 - p2

    def update_height(self, dt):
        """gas_layer_solve.cc:133-162. h[i] is updated in place, so iteration
        i reads the already-updated h[i-1], h[i-2]: a sequential recurrence."""
        m, xsp = self.m, self.prm.xsp
        u0 = self.u[2, 2:2 + m]; ub = self.u[1, 2:2 + m]
        v0 = self.v[2, 2:2 + m]; vb = self.v[1, 2:2 + m]
        uc_all = 0.25 * xsp * (u0 + ub)
        vc_all = 0.5 * (v0 + vb)
        h = self.h
        for i in range(m):
            uc = float(uc_all[i]); vc = float(vc_all[i])
            if uc > 0:
                dhdx = self.eno2(self.h_ref(i + 1), h[i], self.h_ref(i - 1), self.h_ref(i - 2))
            else:
                dhdx = -self.eno2(self.h_ref(i - 1), h[i], self.h_ref(i + 1), self.h_ref(i + 2))
            self.ht[i] = -uc * dhdx + vc - self.Vframe
            h[i] += dt * self.ht[i]
            self.fbd[i] += dt * vc
        self.calculate_hx()

    def newton_assemble(self, dtinv):
        """gas_layer_solve.cc:67-126: tridiagonal Newton system (a: sub,
        b: diagonal, c: super, d: minus the residual) and the mean squared
        residual."""
        prm = self.prm
        me = self.me
        h, ht, hx, pg, pg_old = self.h, self.ht, self.hx, self.pg, self.pg_old
        xsp, xxsp = prm.xsp, prm.xxsp
        mu, alpha, Pamb = prm.mug, prm.alpha, prm.Pamb
        a = np.zeros(me); b = np.zeros(me); c = np.zeros(me); d = np.zeros(me)
        hcu_0 = h[0] * h[0] * h[0]
        if prm.x_sym:
            b[0] = -12 * mu * (alpha * dtinv * h[0] + ht[0]) + 2 * xxsp * hcu_0 * (pg[1] - pg[0]) \
                - 2 * xxsp * hcu_0 * pg[0] - 2 * xxsp * hcu_0 * Pamb
            c[0] = 2 * xxsp * hcu_0 * pg[0] + 2 * xxsp * hcu_0 * Pamb
            d[0] = 12 * mu * (alpha * dtinv * h[0] * (pg[0] - pg_old[0]) + ht[0] * pg[0] + ht[0] * Pamb) \
                - 2 * xxsp * hcu_0 * pg[0] * (pg[1] - pg[0]) - 2 * xxsp * hcu_0 * Pamb * (pg[1] - pg[0])
        else:
            b[0] = 1.; c[0] = 0.; d[0] = -pg[0]
        a[me - 1] = 0.; b[me - 1] = 1.; d[me - 1] = -pg[me - 1]
        i0 = 0 if prm.x_sym else 1
        i = np.arange(i0, me - 1)
        im = np.maximum(i - 1, 0)
        pos = i > 0
        h_ns = np.where(pos, 0.5 * (h[im] + h[i]), h[i])
        ht_ns = np.where(pos, 0.5 * (ht[im] + ht[i]), ht[i])
        px = np.where(pos, 0.5 * xsp * (pg[i + 1] - pg[im]), 0.)
        pxx = np.where(pos, xxsp * (pg[i + 1] - 2 * pg[i] + pg[im]),
                       xxsp * (pg[i + 1] - 2 * pg[i] + pg[i + 1]))
        hsq = h_ns * h_ns
        hcu = hsq * h_ns
        hxi = hx[i]; pgi = pg[i]
        br = 3 * hsq * hxi * px + hcu * pxx - 12 * mu * alpha * h_ns * dtinv - 12 * mu * ht_ns
        ai = -xsp * alpha * hcu * px + pgi * (-1.5 * xsp * hsq * hxi + hcu * xxsp) \
            + Pamb * (-1.5 * xsp * hsq * hxi + hcu * xxsp)
        bi = br - 2 * pgi * hcu * xxsp - 2 * Pamb * hcu * xxsp
        ci = xsp * alpha * hcu * px + pgi * (1.5 * xsp * hsq * hxi + hcu * xxsp) \
            + Pamb * (1.5 * xsp * hsq * hxi + hcu * xxsp)
        ci = np.where(i == 0, ci + ai, ci)
        di = -(12 * mu * alpha * h_ns * dtinv * pg_old[i] + alpha * hcu * px * px + pgi * br
               + Pamb * (-12 * mu * ht_ns + 3 * hsq * hxi * px + hcu * pxx))
        a[i] = ai; b[i] = bi; c[i] = ci; d[i] = di
        ressq = 0.
        for q in di:
            ressq += q * q
        return a, b, c, d, ressq / me

    def newton_step(self, dtinv):
        """gas_layer_solve.cc:67-129 with tri_solve::solve_lapack
        (tri_solve.cc:24-33)."""
        a, b, c, d, res = self.newton_assemble(dtinv)
        x, info = dgtsv(a[1:], b, c[:-1], d)
        if info != 0:
            raise OracleError("LAPACK routine failed")
        self.pg += x
        return res

    def implicit_step(self, dt):
        """gas_layer_solve.cc:197-212."""
        dtinv = 1. / dt
        nstep = naccept = 0
        while naccept < 2:
            nstep += 1
            if nstep > MAX_NEWTON_STEPS:
                raise OracleError("Too many Newton steps")
            if self.newton_step(dtinv) < NEWTON_THRESH:
                naccept += 1
            else:
                naccept = 0
        self.newton_iters.append(nstep)

    def calculate_liquid_fields(self):
        """gas_layer_solve.cc:229-249."""
        prm = self.prm
        m, h, pg, p = self.m, self.h, self.pg, self.gp
        fac = 0.5 * prm.sigma * prm.xxsp
        fac2 = prm.sigma / prm.R
        if prm.x_sym:
            p[0] = pg[0] + 2 * fac * (h[1] - h[0]) - fac2
            p[1] = pg[1] + fac * (h[2] - h[1]) - fac2
        else:
            p[0] = pg[0]; p[1] = pg[1]
        i = np.arange(2, m - 1)
        p[i] = pg[i] + fac * (h[i + 1] - h[i] - h[i - 1] + h[i - 2]) - fac2
        p[m - 1] = pg[m - 1]; p[m] = pg[m]
        self.tau[0:m] = -0.5 * prm.xsp * prm.mug * (p[1:m + 1] - p[0:m]) * h

    def apply_tau_bc(self):
        """gas_layer.cc:25-30."""
        t, ml = self.tau, self.ml
        t[0] = -t[3]; t[1] = -t[2]; t[ml - 2] = -t[ml - 3]; t[ml - 1] = -t[ml - 4]

    def gas_update(self, dt):
        """gas_layer::update (gas_layer.cc:36-46) with
        gas_layer_solve::calc_p_and_tau (gas_layer_solve.cc:215-226)."""
        self.gp_old[:] = self.gp
        self.tau_old[:] = self.tau
        self.update_height(dt)
        self.pg_old[:] = self.pg
        self.implicit_step(dt)
        self.calculate_liquid_fields()
        self.apply_tau_bc()

    # -------------------------------------------------- boundaries
    def simpsons(self, x, y, prefac):
        """fluid_2d_sio.cc:366-405 for arrays of points (x, y): returns the
        increments of (u, v)."""
        prm = self.prm
        me = self.me
        xms = x - prm.ax
        xps = x + prm.ax
        ysq = y * y
        pp = self.gp

        def terms(xms, xps, p):
            rm = xms * xms + ysq
            rm = 1 / (rm * rm)
            if prm.x_sym:
                rp = xps * xps + ysq
                rp = 1 / (rp * rp)
                return p * (xms * rm + xps * rp), -p * ((xms * xms - ysq) * rm + (xps * xps - ysq) * rp)
            return p * xms * rm, -p * (xms * xms - ysq) * rm

        su, sv = terms(xms, xps, pp[0])
        xms = xms - prm.dx; xps = xps + prm.dx
        for j in range(1, me - 1):
            fsu, fsv = terms(xms, xps, pp[j])
            fac = 4. if (j & 1) else 2.
            su = su + fac * fsu; sv = sv + fac * fsv
            xms = xms - prm.dx; xps = xps + prm.dx
        fsu, fsv = terms(xms, xps, pp[me - 1])
        su = su + fsu; sv = sv + fsv
        return 2 * y * prefac * su, prefac * sv

    def set_inviscid_boundaries(self, dt):
        """fluid_2d_sio.cc:256-290."""
        prm = self.prm
        m, n, ml = self.m, self.n, self.ml
        prefac = prm.dx * prm.rhoinv * dt / (3 * math.pi)
        jj = np.arange(n)
        y = prm.ay + (jj + 0.5) * prm.dy
        du1, dv1 = self.simpsons(np.full(n, prm.bx + prm.dx * 0.5), y, prefac)
        du2, dv2 = self.simpsons(np.full(n, prm.bx + prm.dx * 1.5), y, prefac)
        u, v = self.u, self.v
        r = slice(2, 2 + n)
        u[r, m + 2] += du1; v[r, m + 2] += dv1
        u[r, m + 3] += du2; v[r, m + 3] += dv2
        if not prm.x_sym:
            u[r, 1] = -u[r, m + 2]; v[r, 1] = v[r, m + 2]
            u[r, 0] = -u[r, m + 3]; v[r, 0] = v[r, m + 3]
        ii = np.arange(ml)
        x = prm.ax + (ii - 1.5) * prm.dx
        du1, dv1 = self.simpsons(x, np.full(ml, prm.by + prm.dy * 0.5), prefac)
        du2, dv2 = self.simpsons(x, np.full(ml, prm.by + prm.dy * 1.5), prefac)
        u[n + 2, :] += du1; v[n + 2, :] += dv1
        u[n + 3, :] += du2; v[n + 3, :] += dv2

    def set_viscous_boundaries(self):
        """fluid_2d_sio.cc:294-343 (the tau array is indexed with the +2
        ghost offset, as the reference does)."""
        prm = self.prm
        m, n, ml = self.m, self.n, self.ml
        u, v = self.u, self.v
        if prm.x_sym:
            r = slice(2, 2 + n)
            u[r, 1] = -u[r, 2]; v[r, 1] = v[r, 2]
            u[r, 0] = -u[r, 3]; v[r, 0] = v[r, 3]
        un_edge = prm.muinv * self.tau
        u[1, :] = u[2, :] - prm.dy * un_edge
        u[0, :] = u[3, :] - 3 * prm.dy * un_edge
        c = np.arange(1, m + 2)
        uxa = 0.5 * prm.xsp * (u[1, c + 1] - u[1, c - 1])
        uxb = 0.5 * prm.xsp * (u[0, c + 1] - u[0, c - 1])
        v[1, c] = v[2, c] + prm.dy * uxa
        v[0, c] = v[1, c] + prm.dy * uxb

    def set_boundaries(self, dt):
        """fluid_2d.cc:485-492."""
        self.set_inviscid_boundaries(dt)
        self.set_viscous_boundaries()

    # -------------------------------------------------- solvers
    def _solver(self, key, build):
        s = self._solvers.get(key)
        if s is None:
            s = DirectSolver(build())
            self._solvers[key] = s
        return s

    def solve_mac(self, src):
        prm = self.prm
        return self._solver('mac', lambda: mac_matrix(self.m, self.n, prm.xxsp, prm.yysp)).solve(src.ravel()).reshape(self.n, self.m)

    def solve_fem(self, src):
        prm = self.prm
        return self._solver('fem', lambda: fem_matrix(self.me, self.ne, prm.dx, prm.dy)).solve(src.ravel()).reshape(self.ne, self.me)

    def solve_visco(self, src, vfx, vfy, horizontal):
        prm = self.prm
        return self._solver(('visc', vfx, vfy, horizontal),
                            lambda: visco_matrix(self.m, self.n, vfx, vfy, prm.x_sym, horizontal)
                            ).solve(src.ravel()).reshape(self.n, self.m)

    # -------------------------------------------------- one timestep
    def step(self, dt):
        """fluid_2d::step_forward (fluid_2d.cc:93-405)."""
        prm = self.prm
        m, n, S = self.m, self.n, self.S
        dx, dy, xsp, ysp, xxsp, yysp = prm.dx, prm.dy, prm.xsp, prm.ysp, prm.xxsp, prm.yysp
        u, v, p = self.u, self.v, self.p
        shp = u.shape

        # tracers (fluid_2d.cc:98), then the gas layer (fluid_2d.cc:96-102)
        self.update_tracers(dt)
        self.gas_update(dt)
        self.time += 0.5 * dt

        # stage 1: limited slopes and edge extrapolation (fluid_2d.cc:105-132)
        uy = ysp * mono_diff(S(u, 0, -2), S(u, 0, -1), S(u), S(u, 0, 1), S(u, 0, 2))
        vy = ysp * mono_diff(S(v, 0, -2), S(v, 0, -1), S(v), S(v, 0, 1), S(v, 0, 2))
        ux = xsp * mono_diff(S(u, -2), S(u, -1), S(u), S(u, 1), S(u, 2))
        vx = xsp * mono_diff(S(v, -2), S(v, -1), S(v), S(v, 1), S(v, 2))
        uc, vc = S(u), S(v)
        E = {k: np.zeros(shp) for k in ('ud', 'vd', 'ul', 'vl', 'ur', 'vr', 'uu', 'vu')}
        S(E['ud'])[:] = uc - 0.5 * (dy + dt * vc) * uy
        S(E['vd'])[:] = vc - 0.5 * (dy + dt * vc) * vy
        S(E['ul'])[:] = uc - 0.5 * (dx + dt * uc) * ux
        S(E['vl'])[:] = vc - 0.5 * (dx + dt * uc) * vx
        S(E['ur'])[:] = uc + 0.5 * (dx - dt * uc) * ux
        S(E['vr'])[:] = vc + 0.5 * (dx - dt * uc) * vx
        S(E['uu'])[:] = uc + 0.5 * (dy - dt * vc) * uy
        S(E['vu'])[:] = vc + 0.5 * (dy - dt * vc) * vy

        # stage 2: tangential upwinding (fluid_2d.cc:136-150)
        self._zero_edge(E)
        self._godunov_edges(E, tang=True)

        # stage 3: transverse derivative terms (fluid_2d.cc:153-160)
        ul, vl, ur, vd, ud, vu = E['ul'], E['vl'], E['ur'], E['vd'], E['ud'], E['vu']
        c0 = 0.5 * xsp * (S(ul, 1) + S(ul)) * (S(ur) - S(ur, -1))
        c1 = 0.5 * xsp * (S(ul, 1) + S(ul)) * (S(vl, 1) - S(vl))
        c2 = 0.5 * ysp * (S(vd, 0, 1) + S(vd)) * (S(ud, 0, 1) - S(ud))
        c3 = 0.5 * ysp * (S(vd, 0, 1) + S(vd)) * (S(vu) - S(vu, 0, -1))

        # stage 4: half-step edge velocities (fluid_2d.cc:164-201)
        viscfac = prm.rhoinv * prm.mu * 0.5 if prm.implicit_visc else prm.rhoinv * prm.mu
        px = 0.5 * xsp * (S(p, 1, 1) + S(p, 1) - S(p, 0, 1) - S(p))
        py = 0.5 * ysp * (S(p, 1, 1) - S(p, 1) + S(p, 0, 1) - S(p))
        uyy = yysp * (S(u, 0, -1) - 2 * uc + S(u, 0, 1))
        vyy = yysp * (S(v, 0, -1) - 2 * vc + S(v, 0, 1))
        uxx = xxsp * (S(u, -1) - 2 * uc + S(u, 1))
        vxx = xxsp * (S(v, -1) - 2 * vc + S(v, 1))
        rhoinv = prm.rhoinv
        f_x = -px * rhoinv + viscfac * (uxx + uyy)
        f_y = -py * rhoinv + viscfac * (vxx + vyy)
        S(E['ud'])[:] = uc + 0.5 * (-dy * uy + dt * (-c0 - vc * uy + f_x))
        S(E['vd'])[:] = vc + 0.5 * (-dy * vy + dt * (-c1 - vc * vy + f_y))
        S(E['ul'])[:] = uc + 0.5 * (-dx * ux + dt * (-uc * ux - c2 + f_x))
        S(E['vl'])[:] = vc + 0.5 * (-dx * vx + dt * (-uc * vx - c3 + f_y))
        S(E['ur'])[:] = uc + 0.5 * (dx * ux + dt * (-uc * ux - c2 + f_x))
        S(E['vr'])[:] = vc + 0.5 * (dx * vx + dt * (-uc * vx - c3 + f_y))
        S(E['uu'])[:] = uc + 0.5 * (dy * uy + dt * (-c0 - vc * uy + f_x))
        S(E['vu'])[:] = vc + 0.5 * (dy * vy + dt * (-c1 - vc * vy + f_y))
        fc0 = viscfac * (uxx + uyy)
        fc1 = viscfac * (vxx + vyy)

        # stage 5: normal upwinding (fluid_2d.cc:205-215)
        self._zero_edge(E)
        self._godunov_edges(E, tang=False)

        # MAC source and bottom Dirichlet term (fluid_2d.cc:218-232)
        src = xsp * (S(ul, 1) - S(ul)) + ysp * (S(vd, 0, 1) - S(vd))
        macfac = 0.125 * rhoinv * dt
        gp, gpo = self.gp, self.gp_old
        s_bc = macfac * (gpo[0:m] + gpo[1:m + 1] + gp[0:m] + gp[1:m + 1])
        src[0, :] -= 2 * yysp * s_bc
        q = self.solve_mac(src)
        self.last_mac = (src, q)

        # MAC correction (fluid_2d.cc:236-248)
        S(ul)[:, 1:] -= (q[:, 1:] - q[:, :-1]) * xsp
        S(vd)[1:, :] -= (q[1:, :] - q[:-1, :]) * ysp
        S(vd)[0, :] -= 2 * ysp * (q[0, :] - s_bc)
        self.time += 0.5 * dt

        # advective update (fluid_2d.cc:253-261)
        vl = E['vl']
        fc0 = uc + dt * (-0.5 * (xsp * (S(ul, 1) + S(ul)) * (S(ul, 1) - S(ul))
                                 + ysp * (S(vd, 0, 1) + S(vd)) * (S(ud, 0, 1) - S(ud))) + fc0)
        fc1 = vc + dt * (-0.5 * (xsp * (S(ul, 1) + S(ul)) * (S(vl, 1) - S(vl))
                                 + ysp * (S(vd, 0, 1) + S(vd)) * (S(vd, 0, 1) - S(vd))) + fc1)
        fc0 = fc0.copy(); fc1 = fc1.copy()

        self.set_boundaries(dt)

        # implicit viscosity (fluid_2d.cc:272-335)
        if prm.implicit_visc:
            vfx = viscfac * xxsp * dt
            vfy = viscfac * yysp * dt
            su = fc0.copy()
            if not prm.x_sym:
                su[:, 0] += vfx * u[2:2 + n, 1]
            su[:, m - 1] += vfx * u[2:2 + n, m + 2]
            su[n - 1, :] += vfy * u[n + 2, 2:2 + m]
            dudy = prm.muinv * 0.5 * (self.tau_old[2:2 + m] + self.tau[2:2 + m])
            su[0, :] -= vfy * dy * dudy
            zu = self.solve_visco(su, vfx, vfy, True)
            sv = fc1.copy()
            if not prm.x_sym:
                sv[:, 0] += vfx * v[2:2 + n, 1]
            sv[:, m - 1] += vfx * v[2:2 + n, m + 2]
            sv[n - 1, :] += vfy * v[n + 2, 2:2 + m]
            dvdy = -0.5 * xsp * (u[2, 3:3 + m] - u[2, 1:1 + m])
            sv[0, :] -= vfy * dy * dvdy
            zv = self.solve_visco(sv, vfx, vfy, False)
            self.last_visc = (su, zu, sv, zv)
            fc0, fc1 = zu, zv

        # FEM source (fluid_2d.cc:337-377)
        me, ne = self.me, self.ne
        C0 = np.zeros((n + 1, m + 2)); C1 = np.zeros((n + 1, m + 2))
        # C[jj, ii] holds cell (ii-1, jj) so that node (i, j) reads cells
        # (i-1, j-1), (i-1, j), (i, j-1), (i, j)
        C0[:n, 1:m + 1] = fc0; C1[:n, 1:m + 1] = fc1
        fsrc = np.zeros((ne, me))
        jn = np.arange(1, ne)[:, None]
        inode = np.arange(me)[None, :]
        bl0, bl1 = C0[0:n, 0:me], C1[0:n, 0:me]
        tl0, tl1 = C0[1:n + 1, 0:me], C1[1:n + 1, 0:me]
        br0, br1 = C0[0:n, 1:me + 1], C1[0:n, 1:me + 1]
        tr0, tr1 = C0[1:n + 1, 1:me + 1], C1[1:n + 1, 1:me + 1]
        nl = inode != 0
        nr = inode != m
        top = jn < n
        spx = np.zeros((n, me)); spy = np.zeros((n, me))
        spx = spx + np.where(nl, bl0, 0.); spy = spy + np.where(nl, bl1, 0.)
        spx = spx + np.where(nl & top, tl0, 0.); spy = spy - np.where(nl & top, tl1, 0.)
        spx = spx - np.where(nr, br0, 0.); spy = spy + np.where(nr, br1, 0.)
        spx = spx - np.where(nr & top, tr0, 0.); spy = spy - np.where(nr & top, tr1, 0.)
        fsrc[1:, :] = 0.5 * (dy * spx + dx * spy) * prm.rho / dt
        fl = 0.25 * dy * prm.rho / dt
        for j in range(1, ne):
            if not prm.x_sym:
                if j < n:
                    fsrc[j, 0] += fl * (fc0[j, 0] + u[j + 2, 1])
                fsrc[j, 0] += fl * (fc0[j - 1, 0] + u[j + 1, 1])
        for j in range(1, ne):
            if j < n:
                fsrc[j, m] -= fl * (fc0[j, m - 1] + u[j + 2, m + 2])
            fsrc[j, m] -= fl * (fc0[j - 1, m - 1] + u[j + 1, m + 2])
        ft = 0.25 * dx * prm.rho / dt
        for i in range(me):
            if i > 0:
                fsrc[n, i] -= ft * (fc1[n - 1, i - 1] + v[n + 2, i + 1])
            if i < m:
                fsrc[n, i] -= ft * (fc1[n - 1, i] + v[n + 2, i + 2])
        fcoef = fem_coeffs(dx, dy)
        ii = np.arange(me)
        fsrc[0, :] = fem_a_cc(me, ne, ii, 0, fcoef['fm']) * self.gp
        z = self.solve_fem(fsrc)
        self.last_fem = (fsrc, z)

        # velocity and pressure update (fluid_2d.cc:383-396)
        k = 0.5 * dt * rhoinv * xsp
        kk = 0.5 * dt * rhoinv * ysp
        S(u)[:] = fc0 - k * (z[1:, 1:] + z[:-1, 1:] - z[1:, :-1] - z[:-1, :-1])
        S(v)[:] = fc1 - kk * (z[1:, 1:] - z[:-1, 1:] + z[1:, :-1] - z[:-1, :-1])
        self.N(p)[:] = z

        self.set_viscous_boundaries()
        if prm.nif_mode:
            self.adjust_frame()

    def _zero_edge(self, E):
        """fluid_2d.cc:480-482."""
        if self.prm.x_sym:
            E['ul'][2:2 + self.n, 2] = 0.

    def _godunov_edges(self, E, tang):
        """The edge loops of fluid_2d.cc:137-150 (tang) and 206-215. Every
        edge value is written by one edge only, so the loops vectorise."""
        m, n = self.m, self.n
        r = slice(2, 2 + n)
        ur, ul, vr, vl = E['ur'], E['ul'], E['vr'], E['vl']
        vu, vd, uu, ud = E['vu'], E['vd'], E['uu'], E['ud']
        a = slice(2, 1 + m); b = slice(3, 2 + m)    # cells i=0..m-2 and i+1
        if tang:
            nu0, nu1, nv1 = godunov_set_tang(ur[r, a], ul[r, b], vr[r, a], vl[r, b])
            ur[r, a] = nu0; ul[r, b] = nu1; vl[r, b] = nv1
            ur[r, 1] = ul[r, 2]
        else:
            nu1, nv1 = godunov_set(ur[r, a], ul[r, b], vr[r, a], vl[r, b])
            ul[r, b] = nu1; vl[r, b] = nv1
        ul[r, m + 2] = ur[r, m + 1]; vl[r, m + 2] = vr[r, m + 1]
        c = slice(2, 2 + m)
        ja = slice(2, 1 + n); jb = slice(3, 2 + n)
        if tang:
            nu0, nu1, nv1 = godunov_set_tang(vu[ja, c], vd[jb, c], uu[ja, c], ud[jb, c])
            vu[ja, c] = nu0; vd[jb, c] = nu1; ud[jb, c] = nv1
            vu[1, c] = vd[2, c]
        else:
            nu1, nv1 = godunov_set(vu[ja, c], vd[jb, c], uu[ja, c], ud[jb, c])
            vd[jb, c] = nu1; ud[jb, c] = nv1
        vd[n + 2, c] = vu[n + 1, c]; ud[n + 2, c] = uu[n + 1, c]

    # -------------------------------------------------- state exchange
    def state(self) -> dict:
        return dict(m=self.m, n=self.n, time=self.time, Vframe=self.Vframe,
                    u=self.u.copy(), v=self.v.copy(), p=self.p.copy(),
                    gp=self.gp.copy(), tau=self.tau.copy(), h=self.h.copy(),
                    fbd=self.fbd.copy(), pg=self.pg.copy(), ht=self.ht.copy())

    def load(self, st: dict):
        self.time = float(st['time']); self.Vframe = float(st['Vframe'])
        for k in ('u', 'v', 'p'):
            getattr(self, k)[:] = st[k]
        self.gp[:] = st['gp']; self.tau[:] = st['tau']; self.h[:] = st['h']
        self.fbd[:] = st['fbd']; self.pg[:] = st['pg']; self.ht[:] = st['ht']
        self.calculate_hx()


# --------------------------------------------------------------------------
# State files of oracle/ref_driver.cc
# --------------------------------------------------------------------------
def read_states(path: str) -> list[dict]:
    raw = open(path, 'rb').read()
    out, off = [], 0
    while off < len(raw):
        m, n = np.frombuffer(raw, np.int32, 2, off); off += 8
        m, n = int(m), int(n)
        t, vf = np.frombuffer(raw, np.float64, 2, off); off += 16
        tot = (m + 4) * (n + 4)
        st = dict(m=m, n=n, time=float(t), Vframe=float(vf))
        for k in ('u', 'v', 'p'):
            st[k] = np.frombuffer(raw, np.float64, tot, off).reshape(n + 4, m + 4).copy(); off += 8 * tot
        for k, ln in (('gp', m + 1), ('tau', m + 4), ('h', m), ('fbd', m), ('pg', m + 1), ('ht', m)):
            st[k] = np.frombuffer(raw, np.float64, ln, off).copy(); off += 8 * ln
        out.append(st)
    return out


def write_state(path: str, st: dict):
    with open(path, 'wb') as f:
        f.write(np.array([st['m'], st['n']], np.int32).tobytes())
        f.write(np.array([st['time'], st['Vframe']], np.float64).tobytes())
        for k in ('u', 'v', 'p', 'gp', 'tau', 'h', 'fbd', 'pg', 'ht'):
            f.write(np.ascontiguousarray(st[k], np.float64).tobytes())


def cfg_text(base: str, m: int, n: int, extra: dict | None = None) -> str:
    """A configuration text from a reference .cfg with the grid replaced and
    file output, tracers and timing lines dropped."""
    lines = []
    for raw in base.splitlines():
        key = raw.split('#', 1)[0].split()
        k = key[0] if key else None
        if k in ('grid_points', 'output', 'mr_time_output', 'tracers', 'restart_freq'):
            continue
        if extra and k in extra:
            continue
        lines.append(raw)
    lines.append(f"grid_points {m} {n}")
    lines.append("tracers 0")
    for k, v in (extra or {}).items():
        lines.append(f"{k} {v}")
    return "\n".join(lines) + "\n"
