"""Microstructure data of the temperature field over
include/adamantine_b200_microstructure.h.

Mirrors adamantine::Microstructure (source/Microstructure.hh): the driver
saves the field before a time step (``set_old_temperature``) and collects,
after it, the points where the temperature crossed the liquidus downward
with the thermal gradient G, the cooling rate and R = rate / G
(``compute_G_and_R``). The records are computed on the GPU; with a
filename prefix they are also written to ``<prefix>.txt`` in the reference's
format (one line per record: the coordinates, G, the cooling rate and R,
space separated, 9 significant digits).
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib
from .thermal import ThermalPhysics, _dev


def format_record(r) -> str:
    """One line of the reference's file (std::setprecision(9))."""
    out = []
    for v in r:
        v = float(v)
        if np.isinf(v):
            out.append("inf" if v > 0 else "-inf")
        elif np.isnan(v):
            out.append("-nan" if np.signbit(v) else "nan")
        else:
            out.append("%.9g" % v)
    return " ".join(out)


class Microstructure:
    def __init__(self, physics: ThermalPhysics, filename_prefix: Optional[str] = None):
        self._L = _lib.load()
        self.physics = physics
        h = ctypes.c_void_p()
        _lib.check(self._L.adm_microstructure_create(physics._h, ctypes.byref(h)))
        self._h = h
        self._file = open(filename_prefix + ".txt", "w") if filename_prefix else None
        self._records = np.zeros((0, 6))

    def close(self):
        if self._file is not None:
            self._file.close()
            self._file = None
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.adm_microstructure_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_old_temperature(self, old_temperature: torch.Tensor):
        _lib.check(self._L.adm_microstructure_set_old_temperature(self._h, _dev(old_temperature)))

    def compute_G_and_R(self, temperature: torch.Tensor, delta_t: float) -> np.ndarray:
        """Records (n, 6): x, y, z, G, cooling rate, R, in the reference's
        order; appended to the file when there is one."""
        n = ctypes.c_int64()
        src = _dev(temperature)
        cap = len(self._records)
        buf = self._records if cap else None
        _lib.check(self._L.adm_microstructure_compute_G_and_R(
            self._h, src, float(delta_t), cap, None if buf is None else buf.ctypes.data_as(ctypes.c_void_p),
            ctypes.byref(n)))
        if n.value > cap:
            self._records = np.zeros((n.value, 6))
            _lib.check(self._L.adm_microstructure_compute_G_and_R(
                self._h, src, float(delta_t), n.value, self._records.ctypes.data_as(ctypes.c_void_p),
                ctypes.byref(n)))
        rec = self._records[: n.value].copy()
        if self._file is not None:
            for r in rec:
                self._file.write(format_record(r) + "\n")
            self._file.flush()
        return rec
