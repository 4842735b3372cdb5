"""Anderson acceleration of the closure loop's fixed point, on the device.

``AndersonAccelerator`` has the reference's interface and arithmetic
(orbit/core/closure_iteration.py:568-694): ``update(x_k, g_x_k)``,
``apply_with_safeguard(x_k, g_x_k)``, ``reset()``.  The iterates and
residuals (the flattened closure state, e.g. an OH field over all bins) stay
in HBM as device tensors; the difference vectors, their dot products and the
new iterate are formed by ``orbit_vec_dots`` / ``orbit_vec_combine``: the
residual differences are orthonormalised on the device (classical
Gram-Schmidt with one reorthogonalisation), and only their m x m triangular
factor moves to the host, where its SVD gives the least-squares solution with
the reference's singular-value cutoff (rcond times the largest singular value
of the difference matrix, as np.linalg.lstsq applies it).
Host numpy arrays are accepted and returned as such.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Tuple

import numpy as np

from . import _lib


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def _dots(xs, y) -> np.ndarray:
    out = np.zeros(len(xs))
    _lib.check(_lib.lib().orbit_vec_dots(y.numel(), len(xs), _lib.ptr_array([_lib.ptr(x) for x in xs]),
                                         _lib.ptr(y), out.ctypes.data, _stream()))
    return out


def _combine(coef, xs, beta, y):
    c = np.ascontiguousarray(coef, dtype=np.float64)
    _lib.check(_lib.lib().orbit_vec_combine(y.numel(), len(xs), c.ctypes.data,
                                            _lib.ptr_array([_lib.ptr(x) for x in xs]), float(beta), _lib.ptr(y),
                                            _stream()))
    return y


class AndersonAccelerator:
    def __init__(self, m: int = 3, beta: float = 1.0, rcond: float = 1e-10, safeguard_factor: float = 1.5):
        if m < 1:
            raise ValueError(f"Anderson memory depth m must be >= 1, got {m}")
        if m > 15:
            raise ValueError("the device Anderson step keeps at most 15 differences")
        self.m = int(m)
        self.beta = float(beta)
        self.rcond = float(rcond)
        self.safeguard_factor = float(safeguard_factor)
        self.X: List = []
        self.F: List = []
        self.n_updates = 0
        self.n_safeguard_falls = 0

    def reset(self) -> None:
        self.X.clear()
        self.F.clear()

    @staticmethod
    def _dev(v):
        import torch
        if isinstance(v, torch.Tensor):
            return v.to(device="cuda", dtype=torch.float64).reshape(-1).contiguous(), True
        return torch.as_tensor(np.ascontiguousarray(np.asarray(v, dtype=np.float64).ravel()), device="cuda"), False

    def _lstsq(self, D, r):
        """gamma = argmin || r - D gamma ||, the reference's lstsq with its rcond
        cutoff: D = Q R by classical Gram-Schmidt with one reorthogonalisation on
        the device, then the SVD of the small R on the host gives D's singular
        values and the pseudo-inverse solution."""
        import torch
        k = len(D)
        Q = []
        R = np.zeros((k, k))
        for j in range(k):
            v = D[j].clone()
            for _ in range(2):
                if Q:
                    h = _dots(Q, v)
                    _combine(list(-h), Q, 1.0, v)
                    R[:j, j] += h
            nrm = float(np.sqrt(max(_dots([v], v)[0], 0.0)))
            R[j, j] = nrm
            q = torch.zeros_like(v) if nrm == 0.0 else _combine([1.0 / nrm], [v], 0.0, torch.empty_like(v))
            Q.append(q)
        qr = _dots(Q, r)
        U, sig, Vt = np.linalg.svd(R)
        keep = sig > self.rcond * sig.max() if sig.max() > 0 else np.zeros(k, bool)
        return Vt[keep].T @ ((U[:, keep].T @ qr) / sig[keep])

    def _update(self, x, g):
        import torch
        r = g.clone()
        _combine([-1.0], [x], 1.0, r)  # r = g - x
        self.X.append(x.clone())
        self.F.append(r.clone())
        while len(self.X) > self.m + 1:
            self.X.pop(0)
            self.F.pop(0)
        self.n_updates += 1
        k = len(self.F) - 1
        if k == 0:
            return _combine([self.beta], [r], 1.0, x.clone()), r, None
        DF = [_combine([1.0, -1.0], [self.F[i + 1], self.F[i]], 0.0, torch.empty_like(x)) for i in range(k)]
        DX = [_combine([1.0, -1.0], [self.X[i + 1], self.X[i]], 0.0, torch.empty_like(x)) for i in range(k)]
        gamma = self._lstsq(DF, r)
        # x + beta r - (DX + beta DF) gamma
        xn = _combine([self.beta] + list(-gamma) + list(-self.beta * gamma), [r] + DX + DF, 1.0, x.clone())
        return xn, r, (DF, gamma)

    def update(self, x_k, g_x_k):
        x, is_t = self._dev(x_k)
        g, _ = self._dev(g_x_k)
        xn, _, _ = self._update(x, g)
        return xn if is_t else xn.cpu().numpy()

    def apply_with_safeguard(self, x_k, g_x_k) -> Tuple[object, bool]:
        x, is_t = self._dev(x_k)
        g, _ = self._dev(g_x_k)
        snap_X = [a.clone() for a in self.X]
        snap_F = [a.clone() for a in self.F]
        xn, r, ls = self._update(x, g)
        if ls is None:
            return (xn if is_t else xn.cpu().numpy()), True
        DF, gamma = ls
        res = _combine(list(-gamma), DF, 1.0, r.clone())  # r - DF gamma
        proj = float(np.sqrt(max(_dots([res], res)[0], 0.0)))
        if proj > self.safeguard_factor * float(np.sqrt(max(_dots([r], r)[0], 0.0))):
            self.X, self.F = snap_X, snap_F
            self.reset()
            self.n_safeguard_falls += 1
            xp = _combine([self.beta], [r], 1.0, x.clone())
            return (xp if is_t else xp.cpu().numpy()), False
        return (xn if is_t else xn.cpu().numpy()), True

    def __repr__(self) -> str:
        return (f"AndersonAccelerator(m={self.m}, beta={self.beta}, history_len={len(self.X)}, "
                f"updates={self.n_updates}, safeguard_falls={self.n_safeguard_falls})")
