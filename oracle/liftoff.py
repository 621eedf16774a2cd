"""ORACLE TEST INFRASTRUCTURE — not part of the product.

A CPU restatement, in numpy, of the reference's lift-off analysis
(tt_analysis.cc): Gaussian smoothing of a height profile, the minimum of its
piecewise cubic Hermite interpolant, and the search over successive states
for the global minimum height (lift-off) and the evanescent-field time origin.

The reference reads float32 Gnuplot files (gas_layer_solve.cc:258-282) and
mixes float and double arithmetic; the restatement keeps each of those
roundings so that its per-state output matches the reference tool's printed
digits. Two behaviours of the reference are fixed here:
  - the tangent t1 of the last interval reads q[m], one past the smoothed
    profile (tt_analysis.cc:119, whose k == m-1 branch is never taken); the
    restatement reads 0 there;
  - the tool analyses saved frames; the same analysis applied after every
    timestep (index k, interval dt) is the per-step lift-off search.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

F32 = np.float32
H_EV = float(F32(500e-9))        # tt_analysis.cc:16
GLEN = F32(1.2e-6)               # tt_analysis.cc:19
GAUSSIAN_FAC = F32(7.0)          # tt_analysis.cc:23


def hermite(x, t0, t1, t2, t3):
    """tt_analysis.cc:29-31."""
    return t0 * x * x * (3 - 2 * x) + x * (1 - x) * (-t1 * (1 - x) + t2 * x) + t3 * (2 * x * x * x - 3 * x * x + 1)


def gaussian_weights(dx: float):
    """The normalised weights sp2[-cut..cut] of smooth() (tt_analysis.cc:37-47),
    with its float32 variables (sls, fac, v) and double weights."""
    sls = F32(float(GLEN) / dx)
    fac = F32(0.5 / float(sls * sls))
    cut = int(sls * GAUSSIAN_FAC) + 1
    w = np.zeros(cut + 1)
    v = F32(0.5)
    for i in range(1, cut + 1):
        w[i] = math.exp(float(F32(F32(-fac * F32(i)) * F32(i))))
        v = F32(float(v) + w[i])
    v = F32(0.5 / float(v))
    w[0] = float(v)
    w[1:] = w[1:] * float(v)
    return np.concatenate([w[:0:-1], w]), cut


def smooth(f: np.ndarray, dx: float) -> np.ndarray:
    """tt_analysis.cc:36-57: q[i] = sum_j w[j-i] f[reflect(j)] accumulated in
    a float32 variable, with even reflection at both ends."""
    m = f.size
    w, cut = gaussian_weights(dx)
    idx = np.arange(m)
    v = np.zeros(m, dtype=F32)
    for off in range(-cut, cut + 1):
        j = idx + off
        j = np.where(j < 0, -1 - j, np.where(j >= m, 2 * m - 1 - j, j))
        v = (v.astype(np.float64) + w[off + cut] * f[j]).astype(F32)
    return v.astype(np.float64)


def profile_min(f: np.ndarray, x: np.ndarray, dx: float, smoothed: bool = True):
    """(xmin, fmin) of one height profile (tt_analysis.cc:111-146). f and x
    are the float32 values of the Gnuplot file, widened to double."""
    m = f.size
    q = smooth(f, dx) if smoothed else f.astype(np.float64)
    qe = np.concatenate([q, [0.0]])             # q[m]: see the module docstring
    fmin, xmin = float(f[0]), float(x[0])
    for k in range(m - 1):
        f0, f1, f2 = qe[k], qe[k + 1], qe[k + 2]
        t0 = f1
        t1 = 0.5 * (f2 - f0)
        t2 = (f1 - f0) if k == 0 else 0.5 * (f1 - qe[k - 1])
        t3 = f0
        a = 6 * (t3 - t0) + 3 * (t1 + t2)
        b = 6 * t0 - 2 * t1 - 4 * t2 - 6 * t3
        c = t2
        det = b * b - 4 * a * c
        if f1 < fmin:
            fmin, xmin = f1, float(x[k + 1])
        if smoothed and det >= 0:
            det = math.sqrt(det)
            for r in (0.5 * (-b + det), 0.5 * (-b - det)):
                if 0 < r < a:
                    r /= a
                    fv = hermite(r, t0, t1, t2, t3)
                    if fv < fmin:
                        fmin, xmin = fv, (1 - r) * float(x[k]) + r * float(x[k + 1])
    return xmin, fmin


@dataclass
class LiftoffSearch:
    """The search over successive states (tt_analysis.cc:94-171). interval is
    the time between states (t_end/nframes for frames, dt for steps); R, V,
    h0 are the drop radius, speed and initial height."""
    interval: float
    R: float
    V: float
    h0: float
    gfmin: float = math.inf
    gimin: int = -1
    hsearch: bool = True
    efield: bool = True
    tmin0_ev: float = 0.0
    count: int = 0

    def add(self, xmin: float, fmin: float):
        i = self.count
        if self.hsearch and fmin < self.gfmin:
            self.gfmin, self.gimin = fmin, i
            if self.efield and fmin < H_EV:
                self.tmin0_ev = i * self.interval - xmin * xmin / (2 * self.R * self.V) + H_EV / self.V
                self.efield = False
        if fmin > self.gfmin * 1.005:
            self.hsearch = False
        self.count += 1

    def summary(self):
        """(gfmin, lift-off time - h0/V, lift-off time - evanescent origin,
        percent of states) as the tool's last line prints them."""
        gtmin = self.gimin * self.interval
        pct = 100.0 * float(F32(self.gimin)) / float(F32(self.count - 1))
        return self.gfmin, gtmin - self.h0 / self.V, gtmin - self.tmin0_ev, pct


def analyse(heights, x, dx, interval, R, V, h0, smoothed=True):
    """Runs the search over a sequence of profiles; returns (rows, search)
    with rows[i] = (i, i*interval, xmin, fmin)."""
    s = LiftoffSearch(interval, R, V, h0)
    rows = []
    for i, f in enumerate(heights):
        xm, fm = profile_min(np.asarray(f, dtype=np.float64), x, dx, smoothed)
        rows.append((i, i * interval, xm, fm))
        s.add(xm, fm)
    return rows, s
