"""adm_vmult_host_static: the host-buffer vmult that allocates nothing.

Callers that keep their temperature vectors in host memory and may not
allocate device memory when they apply the operator (for example while a
CUDA graph is being captured elsewhere in the process, or under a device
memory budget fixed at start-up) use this entry point; it stages the vectors
in one static device array instead of cudaMalloc'ed ones. This file is
collected last so that a failure here never hides the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_scratch_vmult_matches_vmult_host():
    from adamantine_b200 import _lib
    from adamantine_b200.thermal import ThermalPhysics
    from pairs import make_case, rel_max

    cfg, cells, T = make_case("q2_slp_goldak")
    g1 = ThermalPhysics(cfg)
    g2 = ThermalPhysics(cfg)
    L = _lib.load()
    assert g2.m() <= 1310720
    g1.set_time(2e-4)
    g2.set_time(2e-4)
    rng = np.random.default_rng(11)
    for call in range(2):
        # two calls in a row: the second must not see the first one's data
        src = g1.to_grid(g1.from_grid(T * (1.0 + 0.03 * call) + rng.uniform(-5, 5, T.shape)))
        src_pad = np.zeros(g1.m())
        src_pad.reshape(g1.nodes[2], g1.nodes[1], g1.pitch)[:, :, : g1.nodes[0]] = src
        ref = g1.vmult_host(src_pad)
        out = np.full(g2.m(), np.nan)
        rc = L.adm_vmult_host_static(g2._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     src_pad.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert rc == 0, L.adm_last_error()
        assert rel_max(out, ref) <= 1e-12
    assert g2.device_error() == 0


def test_static_scratch_rejects_large_meshes():
    from adamantine_b200 import _lib
    from adamantine_b200.thermal import ThermalPhysics
    from adamantine_b200.workloads import phase_change_q2

    g = ThermalPhysics(phase_change_q2(n_cells=(64, 64, 40), extent=(10e-3, 10e-3, 6e-3), powder_layers=8))
    assert g.m() > 1310720
    L = _lib.load()
    buf = np.zeros(g.m())
    rc = L.adm_vmult_host_static(g._h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == 1
    assert b"static staging array" in L.adm_last_error()
