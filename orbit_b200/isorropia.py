"""ISORROPIA 7-D lookup table on the device (the closure loop's partitioning
query).

``IsorropiaLUT(lut_path, fields)`` mirrors the reference class
(orbit/core/isorropia_lut.py:13-147): the table file holds seven ascending
axes (``so4_axis`` ... ``rh_axis``) and float32 fields (``f_nh4``, ``f_no3``,
``aerosol_water``, ``ph``); it is read on the first query and kept in HBM
(float32, as on disk) until ``release()``.  ``query(...)`` takes and returns
host arrays like the reference; ``query_device(pts)`` keeps a (7, n) device
array of points on the device and returns (4, n).  The interpolation runs in
``orbit_lut_query`` (multilinear, linear extrapolation outside the axes, the
reference's output clipping).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib

_AXES = ("so4_axis", "nh_axis", "no3_axis", "ca_axis", "na_axis", "t_axis", "rh_axis")
_FIELDS = ("f_nh4", "f_no3", "aerosol_water", "ph")


class IsorropiaLUT:
    def __init__(self, lut_path, fields=("f_nh4", "f_no3")):
        self._path = str(lut_path)
        self._fields = tuple(fields)
        for f in self._fields:
            if f not in _FIELDS:
                raise ValueError(f"unknown LUT field {f!r}")
        self._dev = None
        self.axes = None
        self.n_loads = 0
        self.load_seconds = 0.0

    def _load(self):
        import torch
        t0 = time.time()
        data = np.load(self._path)
        axes = [np.ascontiguousarray(data[n], dtype=np.float64) for n in _AXES]
        shape = tuple(len(a) for a in axes)
        dev = {"axes": [torch.as_tensor(a, device="cuda") for a in axes], "fields": {}}
        for name in self._fields:
            tab = np.ascontiguousarray(data[name], dtype=np.float32)
            if tab.shape != shape:
                raise ValueError(f"LUT field {name} has shape {tab.shape}, axes give {shape}")
            dev["fields"][name] = torch.as_tensor(tab, device="cuda")
        st = _lib.LutT()
        for d in range(7):
            st.axis[d] = _lib.ptr(dev["axes"][d])
            st.n[d] = shape[d]
        for f, name in enumerate(_FIELDS):
            st.field[f] = _lib.ptr(dev["fields"].get(name))
        dev["struct"] = st
        self._dev = dev
        self.axes = tuple(axes)
        self.n_loads += 1
        self.load_seconds += time.time() - t0

    @property
    def loaded(self):
        return self._dev is not None

    def release(self):
        """Drop the table from HBM; the next query reloads it."""
        self._dev = None

    def query_device(self, pts):
        """pts: (7, n) float64 device tensor -> (4, n) device tensor."""
        import torch
        if self._dev is None:
            self._load()
        pts = pts.to(dtype=torch.float64).contiguous()
        n = pts.shape[1]
        out = torch.empty((4, n), dtype=torch.float64, device=pts.device)
        _lib.check(_lib.lib().orbit_lut_query(C.byref(self._dev["struct"]), n, _lib.ptr(pts), _lib.ptr(out),
                                              torch.cuda.current_stream().cuda_stream))
        return out

    def query(self, total_so4, total_nh, total_no3, crustal_ca, sea_salt_na, T, RH):
        """(f_nh4, f_no3, aerosol_water, ph) at the given points (scalars or
        same-shape arrays, flattened), as the reference returns them."""
        import torch
        cols = [np.atleast_1d(np.asarray(v, dtype=np.float64)).ravel()
                for v in (total_so4, total_nh, total_no3, crustal_ca, sea_salt_na, T, RH)]
        n = max(len(c) for c in cols)
        pts = np.stack([np.broadcast_to(c, (n,)) for c in cols])
        out = self.query_device(torch.as_tensor(np.ascontiguousarray(pts), device="cuda")).cpu().numpy()
        return out[0], out[1], out[2], out[3]
