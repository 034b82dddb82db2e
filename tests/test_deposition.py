"""CPU checks of material deposition: the library's box generation (a host
function of the C ABI) against the reference's known answers and the numpy
restatement, and the activation semantics of the oracle against the
reference's activation tests (test_material_deposition.cc)."""
import os

import numpy as np
import pytest

from deposition_oracle import activate, boxes_along_path, cells_in_box

from adamantine_b200.config import Boundary, Geometry, Source, ThermalConfig
from adamantine_b200.deposition import deposition_boxes, read_material_deposition
from adamantine_b200.workloads import phase_change_material, rng_for, serpentine_segments

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "deposition_inputs.npz"))


def cfg_with_path(seg):
    geo = Geometry(dim=3, n_cells=(4, 4, 4), extent=(1.0, 1.0, 1.0))
    src = Source(type="goldak", depth=1e-4, absorption_efficiency=0.3, diameter=1e-4, max_power=100.0,
                 segments=np.asarray(seg))
    return ThermalConfig(geometry=geo, material=phase_change_material(), boundary=Boundary.from_database(
        {"type": "adiabatic"}, 3), sources=[src], degree=1)


def test_boxes_along_scan_path_known_answers():
    """deposition_from_scan_path_3d (test_material_deposition.cc:443-495)."""
    b = deposition_boxes(cfg_with_path(GOLD["scan_path"]), 0.0005, 0.1, 0.1, 0.0)
    tol = 1e-13
    assert np.allclose(b.lo[0], [-0.00025, 0.05, 0.0], atol=tol, rtol=tol)
    assert np.allclose(b.hi[0], [0.00025, 0.15, 0.1], atol=tol, rtol=tol)
    assert np.allclose(b.lo[4], [0.002 - 0.00025, 0.05, 0.0], atol=tol, rtol=tol)
    assert np.allclose(b.hi[4], [0.002 + 0.00025, 0.15, 0.1], atol=tol, rtol=tol)
    assert np.allclose(b.time[:5], [1.0e-6, 6.26e-4, 1.251e-3, 1.876e-3, 2.501e-3], rtol=tol)
    assert np.all(b.cos[:5] == 1.0) and np.all(b.sin[:5] == 0.0)


def test_boxes_along_L_scan_path_known_answers():
    """deposition_from_L_scan_path_3d (test_material_deposition.cc:497-571)."""
    b = deposition_boxes(cfg_with_path(GOLD["scan_path_L"]), 0.0005, 0.1, 0.1, 0.0)
    tol = 1e-13
    want = {0: ([-0.00025, -0.05, 0.0], [0.00025, 0.05, 0.1]),
            4: ([0.002 - 0.00025, -0.05, 0.0], [0.002 + 0.00025, 0.05, 0.1]),
            5: ([0.002 - 0.05, -0.00025, 0.0], [0.002 + 0.05, 0.00025, 0.1]),
            9: ([0.002 - 0.05, 0.00165, 0.0], [0.002 + 0.05, 0.00195, 0.1])}
    for k, (lo, hi) in want.items():
        assert np.allclose(b.lo[k], lo, atol=tol, rtol=tol), k
        assert np.allclose(b.hi[k], hi, atol=tol, rtol=tol), k
    assert np.allclose(b.time[:10], [1.0e-6, 6.26e-4, 1.251e-3, 1.876e-3, 2.501e-3, 2.501e-3, 3.126e-3, 3.751e-3,
                                     4.376e-3, 0.004751], rtol=tol)


def test_library_boxes_equal_the_restatement():
    seg = serpentine_segments(rng_for("deposition-test"), 1e-3, 9e-3, 2e-3, 5e-3, 6, 300e-6, 1.2)
    b = deposition_boxes(cfg_with_path(seg), 50e-6, 50e-6, 200e-6, 1e-5)
    ref = boxes_along_path(seg, 50e-6, 50e-6, 200e-6, 1e-5)
    order = np.argsort(ref[:, 6], kind="stable")
    ref = ref[order]
    assert b.n == ref.shape[0] > 100
    assert np.array_equal(b.lo, ref[:, 0:3]) and np.array_equal(b.hi, ref[:, 3:6])
    assert np.array_equal(b.time, ref[:, 6])
    assert np.array_equal(b.cos, ref[:, 7]) and np.array_equal(b.sin, ref[:, 8])


def test_cells_in_box_known_answers():
    """get_elements_to_activate_3d (test_material_deposition.cc:195-259):
    12 x 6 x 6 unit cells; the boxes meet 1, 2 and 8 cells."""
    origin, h, nc = (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (12, 6, 6)
    got = [cells_in_box(lo, hi, origin, h, nc) for lo, hi in
           (((0.1, 0.1, 0.1), (0.2, 0.2, 0.2)), ((1.1, 0.1, 0.1), (2.2, 0.2, 0.2)),
            ((4.5, 4.5, 4.5), (5.5, 5.5, 5.5)))]
    assert [g.size for g in got] == [1, 2, 8]
    assert got[0].tolist() == [0]
    assert got[1].tolist() == [1, 2]
    xs = {(c % 12, (c // 12) % 6, c // 72) for c in got[2].tolist()}
    assert xs == {(x, y, z) for x in (4, 5) for y in (4, 5) for z in (4, 5)}


def material_path_case():
    text = "3\n" + "\n".join(" ".join(repr(float(v)) for v in row) for row in GOLD["material_path"])
    boxes = read_material_deposition(text)
    geo = Geometry(dim=3, n_cells=(10, 10, 10), extent=(10.0, 10.0, 10.0), material_height=6.0)
    return boxes, geo


def test_activation_counts_known_answers():
    """material_deposition (test_material_deposition.cc:261-368): the number
    of active cells after each of ten steps of 0.1."""
    boxes, geo = material_path_case()
    active = geo.active_cells().astype(bool)
    assert active.sum() == 600
    dt, t = 0.1, 0.1
    eps = dt / 1e12
    counts = []
    for _ in range(10):
        s = np.searchsorted(boxes.time, t - eps, side="left")
        e = np.searchsorted(boxes.time, t + dt - eps, side="left")
        if s < e:
            cells, _ = activate(active, boxes.lo, boxes.hi, s, e, (0, 0, 0), (1.0, 1.0, 1.0), (10, 10, 10))
            active[cells] = True
        t += dt
        counts.append(int(active.sum()))
    assert counts == [610, 620, 630, 650, 650, 660, 670, 680, 720, 720]
