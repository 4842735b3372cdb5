"""Oracle: the closure loop's ISORROPIA LUT query and Anderson step (numpy).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Restates:

* ``IsorropiaLUT.query``            orbit/core/isorropia_lut.py:116-147
  (scipy RegularGridInterpolator, "linear", fill_value None: multilinear
  inside the axes, linear extrapolation from the edge cells outside; the
  fractions clipped to [0, 1], the water to >= 0)
* ``AndersonAccelerator``           orbit/core/closure_iteration.py:568-694
"""
from __future__ import annotations

import numpy as np


def lut_query(axes, fields, pts):
    """axes: 7 ascending arrays; fields: list of 4 tables (or None); pts (n, 7)."""
    pts = np.asarray(pts, dtype=np.float64)
    n = pts.shape[0]
    idx = np.empty((n, 7), dtype=np.int64)
    t = np.empty((n, 7))
    for d, a in enumerate(axes):
        i = np.clip(np.searchsorted(a, pts[:, d], side="right") - 1, 0, len(a) - 2)
        idx[:, d] = i
        t[:, d] = (pts[:, d] - a[i]) / (a[i + 1] - a[i])
    out = []
    for f, tab in enumerate(fields):
        if tab is None:
            out.append(np.full(n, np.nan))
            continue
        v = np.zeros(n)
        for corner in range(128):
            bits = [(corner >> (6 - d)) & 1 for d in range(7)]
            w = np.ones(n)
            for d in range(7):
                w *= t[:, d] if bits[d] else 1.0 - t[:, d]
            v += w * tab[tuple(idx[:, d] + bits[d] for d in range(7))].astype(np.float64)
        if f < 2:
            v = np.clip(v, 0.0, 1.0)
        elif f == 2:
            v = np.maximum(v, 0.0)
        out.append(v)
    return out


class Anderson:
    """Anderson(m) mixing with the monotonicity safeguard (the reference's
    update / apply_with_safeguard)."""

    def __init__(self, m=3, beta=1.0, rcond=1e-10, safeguard_factor=1.5):
        self.m, self.beta, self.rcond, self.sf = m, beta, rcond, safeguard_factor
        self.X, self.F = [], []

    def update(self, x, g):
        x = np.asarray(x, dtype=np.float64).ravel()
        r = np.asarray(g, dtype=np.float64).ravel() - x
        self.X.append(x.copy())
        self.F.append(r.copy())
        while len(self.X) > self.m + 1:
            self.X.pop(0)
            self.F.pop(0)
        k = len(self.F) - 1
        if k == 0:
            return x + self.beta * r
        DF = np.column_stack([self.F[i + 1] - self.F[i] for i in range(k)])
        DX = np.column_stack([self.X[i + 1] - self.X[i] for i in range(k)])
        gam = np.linalg.lstsq(DF, r, rcond=self.rcond)[0]
        return x + self.beta * r - (DX + self.beta * DF) @ gam

    def apply_with_safeguard(self, x, g):
        x = np.asarray(x, dtype=np.float64).ravel()
        r = np.asarray(g, dtype=np.float64).ravel() - x
        sx, sf = [a.copy() for a in self.X], [a.copy() for a in self.F]
        xn = self.update(x, g)
        if len(self.F) <= 1:
            return xn, True
        k = len(self.F) - 1
        DF = np.column_stack([self.F[i + 1] - self.F[i] for i in range(k)])
        gam = np.linalg.lstsq(DF, r, rcond=self.rcond)[0]
        if np.linalg.norm(r - DF @ gam) > self.sf * np.linalg.norm(r):
            self.X, self.F = sx, sf
            self.X.clear()
            self.F.clear()
            return x + self.beta * r, False
        return xn, True
