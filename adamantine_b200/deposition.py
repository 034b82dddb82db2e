"""Material deposition over include/adamantine_b200_deposition.h.

``deposition_boxes`` builds the boxes along the scan paths of the sources
(deposition_along_scan_path, source/material_deposition.cc:129-324);
``read_material_deposition`` reads a box file (:55-127); ``Deposition`` binds
boxes to a ThermalPhysics and activates the cells they meet on the device,
per box range or with the driver's per-step window
(application/adamantine.hh:1134-1199).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from .config import SourceStruct, ThermalConfig
from .thermal import ThermalPhysics, _dev, _ptr


@dataclass
class Boxes:
    lo: np.ndarray    # (n, 3)
    hi: np.ndarray    # (n, 3)
    time: np.ndarray  # (n,)
    cos: np.ndarray   # (n,)
    sin: np.ndarray   # (n,)

    @property
    def n(self) -> int:
        return int(self.time.size)


def deposition_boxes(config: ThermalConfig, length: float, height: float, width: float = 0.0,
                     lead_time: float = 0.0) -> Boxes:
    """Boxes of length x width x height along the power-on segments of the
    sources of config, in chronological order."""
    L = _lib.load()
    st = config.to_struct()
    n = ctypes.c_int64()
    args = (ctypes.cast(ctypes.byref(st.sources), ctypes.POINTER(SourceStruct)), st.n_sources, float(length),
            float(height), float(width), float(lead_time))
    _lib.check(L.adm_deposition_boxes(*args, 0, None, None, None, None, None, ctypes.byref(n)))
    m = int(n.value)
    b = Boxes(np.zeros((m, 3)), np.zeros((m, 3)), np.zeros(m), np.zeros(m), np.zeros(m))
    if m:
        _lib.check(L.adm_deposition_boxes(*args, m, _ptr(b.lo, ctypes.c_double), _ptr(b.hi, ctypes.c_double),
                                          _ptr(b.time, ctypes.c_double), _ptr(b.cos, ctypes.c_double),
                                          _ptr(b.sin, ctypes.c_double), ctypes.byref(n)))
    return b


def read_material_deposition(text: str) -> Boxes:
    """A box file: the dimension (3), then one box per line: center[3],
    size[3], deposition time, deposition angle (radians)."""
    lines = [ln for ln in text.splitlines() if ln.strip()]
    if int(lines[0]) != 3:
        raise ValueError("only three-dimensional box files are supported")
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[1:]]).reshape(-1, 8)
    if np.any(np.diff(rows[:, 6]) < 0):
        raise ValueError("Time stamp not increasing.")
    c, s = rows[:, :3], rows[:, 3:6]
    return Boxes(c - 0.5 * s, c + 0.5 * s, rows[:, 6].copy(), np.cos(rows[:, 7]), np.sin(rows[:, 7]))


class Deposition:
    """Deposition boxes bound to a set-up ThermalPhysics."""

    def __init__(self, phys: ThermalPhysics, boxes: Boxes, deposition_time: float = 0.0,
                 duration: float = float(np.finfo(np.float64).max)):
        self._L = _lib.load()
        self.phys = phys
        self.boxes = boxes
        self._arr = [np.ascontiguousarray(a, np.float64) for a in (boxes.lo, boxes.hi, boxes.time, boxes.cos,
                                                                   boxes.sin)]
        h = ctypes.c_void_p()
        _lib.check(self._L.adm_deposition_create(phys._h, boxes.n, *[_ptr(a, ctypes.c_double) for a in self._arr],
                                                 float(deposition_time), float(duration), ctypes.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.adm_deposition_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def activate_range(self, b0: int, b1: int, new_temperature: float, solution) -> int:
        n = ctypes.c_int64()
        _lib.check(self._L.adm_deposition_activate_range(self._h, int(b0), int(b1), float(new_temperature),
                                                         _dev(solution), ctypes.byref(n)))
        return int(n.value)

    def step(self, time: float, time_step: float, new_temperature: float, solution) -> int:
        n = ctypes.c_int64()
        _lib.check(self._L.adm_deposition_step(self._h, float(time), float(time_step), float(new_temperature),
                                               _dev(solution), ctypes.byref(n)))
        return int(n.value)
