"""The kernels' reciprocal (Newton-Raphson on the rcp.approx.ftz.f64 estimate)
against CUDA's IEEE division, over the range of rho * c_p and far beyond."""
import ctypes

import numpy as np
import pytest
import torch

from adamantine_b200 import _lib

pytestmark = pytest.mark.gpu


def test_reciprocal_within_one_ulp():
    L = _lib.load()
    fn = L.adm_diag_reciprocal
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    fn.restype = ctypes.c_int
    rng = np.random.default_rng(7)
    x = np.concatenate([10.0 ** rng.uniform(-300, 300, 500_000),
                        -(10.0 ** rng.uniform(-300, 300, 100_000)),
                        rng.uniform(1e5, 1e8, 400_000)])
    xd = torch.from_numpy(x).cuda()
    y = torch.empty_like(xd)
    yr = torch.empty_like(xd)
    assert fn(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(yr.data_ptr()),
              x.size) == 0
    y, yr = y.cpu().numpy(), yr.cpu().numpy()
    ulp = np.abs(y - yr) / np.spacing(np.abs(yr))
    assert ulp.max() <= 1.0
