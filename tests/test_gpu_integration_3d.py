"""The reference's 3-D integration case on the GPU through the C ABI: the
anisotropic demo (deposition along the scan path with the driver's window,
conductivity rotated by the deposition angle, solid / powder / liquid,
Goldak source, forward Euler) for its 100 steps, against the CPU oracle run
the same way (every active node to 1e-9), and against the reference's gold
file (test_integration_3d.cc:112-115) in its own 4-significant-digit format
and deal.II DoF order."""
import numpy as np
import pytest

from dealii_order import dof_to_node
from integration_demo import BOX, DT, DURATION, NEW_T, demo_config, driver_dt, gold_text, run_oracle
from pairs import rel_max

from adamantine_b200.deposition import Deposition, deposition_boxes
from adamantine_b200.thermal import ThermalPhysics

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("schedule", [0, 1])
def test_integration_3d_on_the_gpu(schedule):
    cfg = demo_config()
    boxes = deposition_boxes(cfg, *BOX)
    g = ThermalPhysics(cfg)
    g.set_schedule(schedule)
    dep = Deposition(g, boxes, deposition_time=0.0, duration=DURATION)
    y = g.initialize_dof_vector(300.0)
    t, n = 0.0, 0
    while t < DURATION:
        dt = driver_dt(t, DT, DURATION)
        dep.step(t, dt, NEW_T, y)
        t = g.evolve_one_time_step(t, dt, y)
        n += 1
    assert n == 100 and g.device_error() == 0
    y_ref, active, _, _ = run_oracle(cfg, boxes)
    order = dof_to_node(3, cfg.geometry.n_cells, 2, active=active)
    got = g.to_grid(y).reshape(-1)[order]
    assert rel_max(got, y_ref[order]) <= 1e-9
    gold = np.array([float(v) for v in gold_text()])
    assert len(got) == len(gold) == 26177
    # within the gold's printed precision (half a unit of the 4th digit)
    assert np.all(np.abs(got - gold) <= 0.5e-3 * 10.0 ** np.floor(np.log10(np.abs(gold))) * (1 + 1e-9))


@pytest.mark.parametrize("exact", [False, True])
def test_integration_3d_checkpoint_restart(tmp_path, exact):
    """test_integration_3d.cc:117-165: a checkpoint after 80 of the 100 steps,
    then a restart (fresh handle, fresh deposition window, as the driver
    restarts) ends at the uninterrupted run's temperatures to 1e-10. With the
    reference's restart (cell states broadcast to the points) this holds
    because no point of the demo reaches the solidus."""
    cfg = demo_config()
    boxes = deposition_boxes(cfg, *BOX)

    def run(g, dep, y, t, n_stop):
        n = 0
        while t < DURATION and n < n_stop:
            dt = driver_dt(t, DT, DURATION)
            dep.step(t, dt, NEW_T, y)
            t = g.evolve_one_time_step(t, dt, y)
            n += 1
        return t

    g1 = ThermalPhysics(cfg)
    y1 = g1.initialize_dof_vector(300.0)
    run(g1, Deposition(g1, boxes, deposition_time=0.0, duration=DURATION), y1, 0.0, 1000)

    g2 = ThermalPhysics(cfg)
    y2 = g2.initialize_dof_vector(300.0)
    t = run(g2, Deposition(g2, boxes, deposition_time=0.0, duration=DURATION), y2, 0.0, 80)
    path = str(tmp_path / "test_checkpoint")
    g2.save_checkpoint(path, t, y2)
    g3 = ThermalPhysics(cfg)
    y3 = g3.initialize_dof_vector(0.0)
    t3 = g3.load_checkpoint(path, y3, exact=exact)
    assert t3 == t
    run(g3, Deposition(g3, boxes, deposition_time=0.0, duration=DURATION), y3, t3, 1000)
    assert rel_max(g3.to_grid(y3), g1.to_grid(y1)) <= 1e-10


def test_vtk_output_of_the_demo(tmp_path):
    """PostProcessor.write_thermal_output after the demo's deposition run:
    one hexahedron per cell that carries material (deposited cells
    included), the corner temperatures of the device field, and the .pvd
    record."""
    import base64
    import xml.etree.ElementTree as ET

    from adamantine_b200.postprocessor import PostProcessor

    cfg = demo_config()
    boxes = deposition_boxes(cfg, *BOX)
    g = ThermalPhysics(cfg)
    dep = Deposition(g, boxes, deposition_time=0.0, duration=DURATION)
    y = g.initialize_dof_vector(300.0)
    pp = PostProcessor(g, "demo", str(tmp_path))
    t, n = 0.0, 0
    pp.write_thermal_output(0, t, y)
    while t < DURATION:
        dt = driver_dt(t, DT, DURATION)
        dep.step(t, dt, NEW_T, y)
        t = g.evolve_one_time_step(t, dt, y)
        n += 1
    pp.write_thermal_output(n, t, y)
    pp.write_pvd()
    active = g.active_cells()
    assert active.sum() == cfg.geometry.active_cells().sum() + 12
    root = ET.parse(str(tmp_path / f"demo.{n}.0.vtu")).getroot()
    assert int(root.find(".//Piece").get("NumberOfCells")) == active.sum()
    arr = {el.get("Name"): el for el in root.iter("DataArray")}
    raw = base64.b64decode(arr["temperature"].text)
    T = np.frombuffer(raw[4:], np.float64)
    raw = base64.b64decode(arr["Points"].text)
    P = np.frombuffer(raw[4:], np.float64).reshape(-1, 3)
    geo = cfg.geometry
    step = np.array(geo.extent) / (2 * np.array(geo.n_cells))
    ijk = np.rint((P - np.array(geo.origin)) / step).astype(int)
    grid = g.to_grid(y)
    assert (T == grid[ijk[:, 2], ijk[:, 1], ijk[:, 0]]).all()  # the cells' corner values
    assert T.min() >= 285.0 and T.max() > 400.0
    ds = list(ET.parse(str(tmp_path / "demo.pvd")).getroot().iter("DataSet"))
    assert len(ds) == 2 and float(ds[1].get("timestep")) == t
