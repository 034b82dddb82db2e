"""Failure paths on the GPU, provoked on the host or by bounded waits (no
GPU fault, trap or hang): a bounded mbarrier wait gives up and reports it; a
non-finite temperature sets the sticky device error word and the context
stays usable; invalid inputs are rejected with status codes."""
import ctypes

import numpy as np
import pytest
import torch

from pairs import make_case, make_gpu

from adamantine_b200 import _lib
from adamantine_b200.config import ConfigStruct

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_reports():
    L = _lib.load()
    fn = L.adm_diag_wait_timeout
    fn.argtypes = [ctypes.c_longlong, ctypes.POINTER(ctypes.c_int32)]
    fn.restype = ctypes.c_int
    out = ctypes.c_int32(-1)
    import time

    t0 = time.perf_counter()
    assert fn(2000, ctypes.byref(out)) == 0  # 2 ms of wall time
    assert out.value == 1
    assert time.perf_counter() - t0 < 5.0
    assert fn(0, ctypes.byref(out)) != 0 and fn(2000000, ctypes.byref(out)) != 0
    # the device keeps working afterwards
    x = torch.ones(8, device="cuda") * 2
    assert float(x.sum().item()) == 16.0


def test_nonfinite_temperature_sets_device_error_and_context_survives():
    cfg, cells, T = make_case("q2_slp_goldak")
    g = make_gpu(cfg, cells)
    bad = np.array(T, copy=True)
    bad.reshape(-1)[len(bad.reshape(-1)) // 2] = np.nan
    y = g.from_grid(bad)
    g.evolve_one_time_step(0.0, 1e-6, y)
    assert g.device_error() == 1  # DERR_NONFINITE
    # a fresh handle on the same device works
    g2 = make_gpu(cfg, cells)
    y2 = g2.from_grid(T)
    g2.evolve_one_time_step(0.0, 1e-6, y2)
    assert g2.device_error() == 0
    assert torch.isfinite(y2).all()


def test_invalid_inputs_are_rejected():
    from adamantine_b200._lib import AdmError
    from adamantine_b200.thermal import ThermalPhysics

    cfg, cells, T = make_case("q1_solid_convective_goldak")
    L = _lib.load()
    st = cfg.to_struct()
    bad = ConfigStruct()
    ctypes.memmove(ctypes.byref(bad), ctypes.byref(st), ctypes.sizeof(ConfigStruct))
    bad.degree = 3
    h = ctypes.c_void_p()
    assert L.adm_create(ctypes.byref(bad), 0, None, ctypes.byref(h)) == 3  # unsupported degree
    bad.degree = cfg.degree
    bad.n_cells[0] = 1 << 20
    bad.n_cells[1] = 1 << 20
    assert L.adm_create(ctypes.byref(bad), 0, None, ctypes.byref(h)) == 1  # mesh too large
    g = make_gpu(cfg, cells)
    with pytest.raises(AdmError) as ex:
        g.set_cells(initial_state=np.full(g.n_cells, 7, np.uint8))
    assert ex.value.code == 1
    with pytest.raises(AdmError):
        g.update_beam(5, 1e-4, 0.3, 1e-4, 100.0)
