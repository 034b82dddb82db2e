"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product never does.  The oracle takes the
raw bytes of an ``adm_config`` structure (identical layout to ``orc_config``,
checked by a test), so this module does not depend on the product package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libthermal_oracle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_I64 = ctypes.POINTER(ctypes.c_int64)


def build(force: bool = False) -> str:
    """Compile the oracle library with its Makefile (system g++, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(
        os.path.getmtime(os.path.join(_HERE, f)) for f in ("thermal_oracle.cpp", "thermal_oracle.h")
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_void_p]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        for f in ("orc_n_nodes", "orc_n_cells"):
            getattr(L, f).restype = ctypes.c_int64
            getattr(L, f).argtypes = [ctypes.c_void_p]
        L.orc_n_qp.restype = ctypes.c_int32
        L.orc_n_qp.argtypes = [ctypes.c_void_p]
        L.orc_set_cells.argtypes = [ctypes.c_void_p, _U8, _U8, _U8, _D, _D]
        L.orc_setup.argtypes = [ctypes.c_void_p]
        L.orc_set_domain.argtypes = [ctypes.c_void_p, _U8]
        L.orc_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.orc_vmult.argtypes = [ctypes.c_void_p, _D, _D]
        L.orc_vmult_add.argtypes = [ctypes.c_void_p, _D, _D]
        L.orc_inverse_mass.argtypes = [ctypes.c_void_p, _D]
        L.orc_node_active.argtypes = [ctypes.c_void_p, _U8]
        L.orc_evolve_one_time_step.restype = ctypes.c_double
        L.orc_evolve_one_time_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _D]
        L.orc_set_state_to_material_properties.argtypes = [ctypes.c_void_p]
        L.orc_get_state_from_material_properties.argtypes = [ctypes.c_void_p]
        L.orc_get_cell_state.argtypes = [ctypes.c_void_p, _D]
        L.orc_set_cell_state.argtypes = [ctypes.c_void_p, _D]
        L.orc_get_qp_powder.argtypes = [ctypes.c_void_p, _D]
        L.orc_get_qp_liquid.argtypes = [ctypes.c_void_p, _D]
        L.orc_evaluate_material_properties.argtypes = [ctypes.c_void_p, _D, _D]
        L.orc_mark_has_melted.argtypes = [ctypes.c_void_p, ctypes.c_double, _D, _U8]
        L.orc_activate_cells.argtypes = [ctypes.c_void_p, _I64, ctypes.c_int64, ctypes.c_double, _D, _D, _D]
        L.orc_source_values.argtypes = [ctypes.c_void_p, ctypes.c_int32, _D, ctypes.c_int64, _D]
        L.orc_source_state.argtypes = [ctypes.c_void_p, ctypes.c_int32, _D]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_D) if a is not None else None


def _u8(a):
    return a.ctypes.data_as(_U8) if a is not None else None


class Oracle:
    """CPU restatement of ThermalOperator + ThermalPhysics on a box mesh.

    ``config_struct`` is an ``adm_config`` ctypes structure (or any object with
    the same byte layout).
    """

    def __init__(self, config_struct, active=None, material_id=None, initial_state=None,
                 deposition_cos=None, deposition_sin=None, n_states=None, domain=None):
        self._L = lib()
        self._cfg = config_struct
        self._h = self._L.orc_create(ctypes.addressof(config_struct))
        self.n_nodes = int(self._L.orc_n_nodes(self._h))
        self.n_cells = int(self._L.orc_n_cells(self._h))
        self.n_qp = int(self._L.orc_n_qp(self._h))
        self.n_states = int(config_struct.n_states)
        C = self.n_cells
        arrs = [
            None if active is None else np.ascontiguousarray(active, np.uint8).reshape(C),
            None if material_id is None else np.ascontiguousarray(material_id, np.uint8).reshape(C),
            None if initial_state is None else np.ascontiguousarray(initial_state, np.uint8).reshape(C),
            None if deposition_cos is None else np.ascontiguousarray(deposition_cos, np.float64).reshape(C),
            None if deposition_sin is None else np.ascontiguousarray(deposition_sin, np.float64).reshape(C),
        ]
        self._L.orc_set_cells(self._h, _u8(arrs[0]), _u8(arrs[1]), _u8(arrs[2]), _dp(arrs[3]), _dp(arrs[4]))
        if domain is not None:
            self._keep_domain = np.ascontiguousarray(domain, np.uint8).reshape(C)
            self._L.orc_set_domain(self._h, _u8(self._keep_domain))
        self._L.orc_setup(self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.orc_destroy(h)
            self._h = None

    def set_time(self, t: float):
        self._L.orc_set_time(self._h, float(t))

    def vmult(self, src: np.ndarray) -> np.ndarray:
        src = np.ascontiguousarray(src, np.float64)
        dst = np.zeros(self.n_nodes)
        self._L.orc_vmult(self._h, _dp(dst), _dp(src))
        return dst

    def vmult_add(self, dst: np.ndarray, src: np.ndarray):
        assert dst.flags.c_contiguous and dst.dtype == np.float64
        src = np.ascontiguousarray(src, np.float64)
        self._L.orc_vmult_add(self._h, _dp(dst), _dp(src))

    def inverse_mass(self) -> np.ndarray:
        out = np.zeros(self.n_nodes)
        self._L.orc_inverse_mass(self._h, _dp(out))
        return out

    def node_active(self) -> np.ndarray:
        out = np.zeros(self.n_nodes, np.uint8)
        self._L.orc_node_active(self._h, _u8(out))
        return out

    def evolve_one_time_step(self, t: float, dt: float, y: np.ndarray) -> float:
        assert y.flags.c_contiguous and y.dtype == np.float64
        return float(self._L.orc_evolve_one_time_step(self._h, float(t), float(dt), _dp(y)))

    def set_state_to_material_properties(self):
        self._L.orc_set_state_to_material_properties(self._h)

    def get_state_from_material_properties(self):
        self._L.orc_get_state_from_material_properties(self._h)

    def cell_state(self) -> np.ndarray:
        out = np.zeros(self.n_states * self.n_cells)
        self._L.orc_get_cell_state(self._h, _dp(out))
        return out.reshape(self.n_states, self.n_cells)

    def set_cell_state(self, state: np.ndarray):
        s = np.ascontiguousarray(state, np.float64).reshape(-1)
        self._L.orc_set_cell_state(self._h, _dp(s))

    def qp_powder(self) -> np.ndarray:
        out = np.zeros(self.n_cells * self.n_qp)
        if self.n_states == 3:
            self._L.orc_get_qp_powder(self._h, _dp(out))
        return out.reshape(self.n_cells, self.n_qp)

    def qp_liquid(self) -> np.ndarray:
        out = np.zeros(self.n_cells * self.n_qp)
        if self.n_states > 1:
            self._L.orc_get_qp_liquid(self._h, _dp(out))
        return out.reshape(self.n_cells, self.n_qp)

    def evaluate_material_properties(self, temperature: np.ndarray) -> np.ndarray:
        T = np.ascontiguousarray(temperature, np.float64)
        out = np.zeros(8 * self.n_cells)
        self._L.orc_evaluate_material_properties(self._h, _dp(T), _dp(out))
        return out.reshape(8, self.n_cells)

    def mark_has_melted(self, threshold: float, temperature: np.ndarray) -> np.ndarray:
        T = np.ascontiguousarray(temperature, np.float64)
        out = np.zeros(self.n_cells, np.uint8)
        self._L.orc_mark_has_melted(self._h, float(threshold), _dp(T), _u8(out))
        return out

    def activate_cells(self, cells, new_temperature: float, solution: np.ndarray, cos=None, sin=None):
        cells = np.ascontiguousarray(cells, np.int64)
        cs = None if cos is None else np.ascontiguousarray(cos, np.float64)
        sn = None if sin is None else np.ascontiguousarray(sin, np.float64)
        self._L.orc_activate_cells(self._h, cells.ctypes.data_as(_I64), cells.size, float(new_temperature),
                                   _dp(cs), _dp(sn), _dp(solution))

    def source_values(self, beam: int, points: np.ndarray) -> np.ndarray:
        pts = np.zeros((len(points), 3))
        p = np.asarray(points, np.float64)
        pts[:, : p.shape[1]] = p
        out = np.zeros(len(points))
        self._L.orc_source_values(self._h, int(beam), _dp(pts), len(points), _dp(out))
        return out

    def source_state(self, beam: int) -> np.ndarray:
        out = np.zeros(5)
        self._L.orc_source_state(self._h, int(beam), _dp(out))
        return out
