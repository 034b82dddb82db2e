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


def _static_vmult(L, g, src_pad):
    out = np.full(g.m(), np.nan)
    rc = L.adm_vmult_host_static(g._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 src_pad.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == 0, L.adm_last_error()
    return out


def _padded(g, grid):
    src_pad = np.zeros(g.m())
    src_pad.reshape(g.nodes[2], g.nodes[1], g.pitch)[:, :, : g.nodes[0]] = grid
    return src_pad


def test_static_scratch_allocates_nothing_and_serves_handles_of_different_layouts():
    """The device's free memory does not move across the first call on a
    freshly set-up handle (the library's module, with the static array, was
    loaded by an earlier call), and handles of different node layouts
    (FE_Q(2) and FE_Q(1) meshes of different sizes) take turns on the shared
    array, each matching its own adm_vmult_host."""
    import torch

    from adamantine_b200 import _lib
    from adamantine_b200.thermal import ThermalPhysics
    from pairs import make_case, rel_max

    L = _lib.load()
    cfg2, _, T2 = make_case("q2_slp_goldak")
    cfg1, _, T1 = make_case("q1_solid_convective_goldak")
    warm = ThermalPhysics(cfg2)
    warm.set_time(2e-4)
    _static_vmult(L, warm, _padded(warm, T2))
    ref2, ref1 = ThermalPhysics(cfg2), ThermalPhysics(cfg1)
    a = ThermalPhysics(cfg2)
    b = ThermalPhysics(cfg1)
    assert (a.nodes, a.pitch) != (b.nodes, b.pitch)
    for g in (ref2, ref1, a, b):
        g.set_time(2e-4)
    # the expected outputs first (adm_vmult_host may allocate on its first
    # call), applied in the order the static calls below see the fields
    srcs = [(None, _padded(a, T2))]
    for k in range(2):
        srcs += [(b, _padded(b, T1 * (1.0 + 0.02 * k))), (a, _padded(a, T2 * (1.0 + 0.02 * k)))]
    expected = [(ref2 if g is not b else ref1).vmult_host(sp) for g, sp in srcs]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    got = [_static_vmult(L, a if g is None else g, sp) for g, sp in srcs]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    for out, ref in zip(got, expected):
        assert rel_max(out, ref) <= 1e-12
    assert a.device_error() == 0 and b.device_error() == 0
