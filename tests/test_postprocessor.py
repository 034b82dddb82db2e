"""The VTK writer of adamantine_b200.postprocessor on synthetic fields (CPU):
the files decode to the active cells' corners, their temperatures and the
cell ratios, and the records name the pieces and times."""
import base64
import os
import xml.etree.ElementTree as ET

import numpy as np

from adamantine_b200.postprocessor import write_pvd, write_pvtu_record, write_vtu


def decode(el, dtype, comps=1):
    raw = base64.b64decode(el.text)
    n = np.frombuffer(raw[:4], np.uint32)[0]
    a = np.frombuffer(raw[4:4 + n], dtype)
    return a.reshape(-1, comps) if comps > 1 else a


def arrays(root):
    return {el.get("Name"): el for el in root.iter("DataArray")}


def test_vtu_holds_the_active_cells_and_fields(tmp_path):
    n_cells, extent, origin, deg = (3, 2, 2), (3e-3, 2e-3, 1e-3), (1e-3, 0.0, -1e-3), 2
    nn = [deg * n + 1 for n in n_cells]
    z, y, x = np.meshgrid(*[origin[d] + np.arange(nn[d]) * extent[d] / (deg * n_cells[d]) for d in (2, 1, 0)],
                          indexing="ij")
    T = 300.0 + 1e5 * x + 2e5 * y - 3e4 * z
    active = np.ones(12, np.uint8)
    active[[1, 7]] = 0
    state = np.zeros((3, 12))
    state[0] = np.linspace(0.1, 0.9, 12)
    state[2] = 1.0 - state[0]
    path = str(tmp_path / "out.3.0.vtu")
    write_vtu(path, 1.5e-3, n_cells, extent, origin, deg, T, active, state)
    root = ET.parse(path).getroot()
    a = arrays(root)
    piece = root.find(".//Piece")
    assert int(piece.get("NumberOfCells")) == 10
    pts = decode(a["Points"], np.float64, 3)
    Tp = decode(a["temperature"], np.float64)
    assert np.allclose(Tp, 300.0 + 1e5 * pts[:, 0] + 2e5 * pts[:, 1] - 3e4 * pts[:, 2], rtol=0, atol=1e-9)
    conn = decode(a["connectivity"], np.int64).reshape(-1, 8)
    assert (decode(a["offsets"], np.int64) == np.arange(8, 81, 8)).all()
    assert (decode(a["types"], np.uint8) == 12).all()
    h = np.array(extent) / np.array(n_cells)
    # every hexahedron spans one cell, corners in VTK order
    for c in conn:
        p = pts[c]
        assert np.allclose(p[6] - p[0], h) and np.allclose(p[1] - p[0], [h[0], 0, 0])
        assert np.allclose(p[3] - p[0], [0, h[1], 0]) and np.allclose(p[4] - p[0], [0, 0, h[2]])
    cells = [i for i in range(12) if active[i]]
    assert np.allclose(decode(a["solid"], np.float64), state[0][cells])
    assert np.allclose(decode(a["powder"], np.float64), state[2][cells])
    assert np.allclose(decode(a["liquid"], np.float64), 0.0)
    assert decode(a["TIME"], np.float64)[0] == 1.5e-3


def test_records(tmp_path):
    p = str(tmp_path / "out.3.pvtu")
    write_pvtu_record(p, ["out.3.0.vtu"])
    root = ET.parse(p).getroot()
    assert [e.get("Source") for e in root.iter("Piece")] == ["out.3.0.vtu"]
    q = str(tmp_path / "out.pvd")
    write_pvd(q, [(0.0, "out.0.pvtu"), (1e-3, "out.3.pvtu")])
    ds = list(ET.parse(q).getroot().iter("DataSet"))
    assert [(float(d.get("timestep")), d.get("file")) for d in ds] == [(0.0, "out.0.pvtu"), (1e-3, "out.3.pvtu")]
    assert os.path.exists(q)
