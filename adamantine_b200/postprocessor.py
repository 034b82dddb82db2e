"""VTK output of the thermal fields, mirroring adamantine::PostProcessor
(source/PostProcessor.hh:218-233, PostProcessor.cc:85-90,141-146,175-227).

Per output step the reference writes ``<prefix>.<step>.<rank>.vtu`` with the
nodal temperature and the cell ratios powder / liquid / solid and the
subdomain, the record ``<prefix>.<step>.pvtu`` naming the ranks' pieces, and
at the end ``<prefix>.pvd`` pairing every record with its time. This writer
produces the same files and fields for one process (rank 0) in plain VTK XML
(one hexahedron per active cell with the values at its corners, binary data
base64-encoded), which ParaView and VisIt read; deal.II's own writer adds
subdivisions and compression that do not change the fields.
"""
from __future__ import annotations

import base64
import os
from typing import List, Optional, Tuple

import numpy as np

_VTK_HEXAHEDRON = 12


def _b64(a: np.ndarray) -> str:
    """VTK XML binary data: a UInt32 byte count, then the bytes, base64."""
    raw = np.ascontiguousarray(a).tobytes()
    return base64.b64encode(np.uint32(len(raw)).tobytes() + raw).decode("ascii")


def _array(name: str, a: np.ndarray, vtk_type: str, components: int = 1) -> str:
    return (f'<DataArray type="{vtk_type}" Name="{name}" NumberOfComponents="{components}" '
            f'format="binary">{_b64(a)}</DataArray>')


def hex_mesh(n_cells, extent, origin, degree: int, active: np.ndarray):
    """Points, connectivity and the grid-node index of every point of the
    active cells of a structured box (the cells' corners, VTK vertex order)."""
    nc = [int(n) for n in n_cells]
    nn = [degree * n + 1 for n in nc]
    act = np.asarray(active, bool).reshape(nc[2], nc[1], nc[0])
    cz, cy, cx = np.nonzero(act)
    # VTK hexahedron corners: bottom face counter-clockwise, then top
    corners = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    nodes = np.stack([(degree * (cx + a)) + nn[0] * ((degree * (cy + b)) + nn[1] * (degree * (cz + c)))
                      for a, b, c in corners], axis=1)  # (n_active, 8) grid-node indices
    used, conn = np.unique(nodes.reshape(-1), return_inverse=True)
    h = [float(extent[d]) / nc[d] for d in range(3)]
    i = used % nn[0]
    j = (used // nn[0]) % nn[1]
    k = used // (nn[0] * nn[1])
    pts = np.stack([origin[0] + i * h[0] / degree, origin[1] + j * h[1] / degree, origin[2] + k * h[2] / degree],
                   axis=1)
    cell_ids = cx + nc[0] * (cy + nc[1] * cz)
    return pts, conn.reshape(-1, 8), used, cell_ids


def write_vtu(path: str, time: float, n_cells, extent, origin, degree: int, temperature_grid: np.ndarray,
              active: np.ndarray, state: Optional[np.ndarray] = None, subdomain: int = 0):
    """One piece: temperature_grid of the node shape (z, y, x), active (n_cells,),
    state (n_states, n_cells) ordered solid, liquid, powder (missing states
    written as 0)."""
    pts, conn, used, cells = hex_mesh(n_cells, extent, origin, degree, active)
    T = np.asarray(temperature_grid, np.float64).reshape(-1)[used]
    n_pts, n_hex = len(pts), len(conn)
    st = np.zeros((3, int(np.prod(n_cells))))
    if state is not None:
        s = np.asarray(state, np.float64)
        st[: s.shape[0]] = s
    solid, liquid, powder = st[0][cells], st[1][cells], st[2][cells]
    offsets = np.arange(8, 8 * n_hex + 1, 8, dtype=np.int64)
    types = np.full(n_hex, _VTK_HEXAHEDRON, np.uint8)
    with open(path, "w") as f:
        f.write('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="0.1" '
                'byte_order="LittleEndian" header_type="UInt32">\n<UnstructuredGrid>\n')
        f.write(f'<FieldData>{_array("TIME", np.array([time], np.float64), "Float64")}</FieldData>\n')
        f.write(f'<Piece NumberOfPoints="{n_pts}" NumberOfCells="{n_hex}">\n')
        f.write(f'<Points>{_array("Points", pts.astype(np.float64), "Float64", 3)}</Points>\n')
        f.write('<Cells>' + _array("connectivity", conn.astype(np.int64), "Int64") +
                _array("offsets", offsets, "Int64") + _array("types", types, "UInt8") + '</Cells>\n')
        f.write('<PointData Scalars="temperature">' + _array("temperature", T, "Float64") + '</PointData>\n')
        f.write('<CellData>' + _array("powder", powder, "Float64") + _array("liquid", liquid, "Float64") +
                _array("solid", solid, "Float64") +
                _array("subdomain", np.full(n_hex, subdomain, np.float32), "Float32") + '</CellData>\n')
        f.write('</Piece>\n</UnstructuredGrid>\n</VTKFile>\n')


def write_pvtu_record(path: str, pieces: List[str]):
    with open(path, "w") as f:
        f.write('<?xml version="1.0"?>\n<VTKFile type="PUnstructuredGrid" version="0.1" '
                'byte_order="LittleEndian" header_type="UInt32">\n<PUnstructuredGrid GhostLevel="0">\n')
        f.write('<PPointData Scalars="temperature"><PDataArray type="Float64" Name="temperature"/></PPointData>\n')
        f.write('<PCellData>' + "".join(f'<PDataArray type="Float64" Name="{n}"/>' for n in ("powder", "liquid",
                                                                                          "solid")) +
                '<PDataArray type="Float32" Name="subdomain"/></PCellData>\n')
        f.write('<PPoints><PDataArray type="Float64" NumberOfComponents="3"/></PPoints>\n')
        for p in pieces:
            f.write(f'<Piece Source="{p}"/>\n')
        f.write('</PUnstructuredGrid>\n</VTKFile>\n')


def write_pvd(path: str, times_filenames: List[Tuple[float, str]]):
    with open(path, "w") as f:
        f.write('<?xml version="1.0"?>\n<VTKFile type="Collection" version="0.1" ByteOrder="LittleEndian">\n'
                '<Collection>\n')
        for t, name in times_filenames:
            f.write(f'<DataSet timestep="{t!r}" group="" part="0" file="{name}"/>\n')
        f.write('</Collection>\n</VTKFile>\n')


class PostProcessor:
    """write_thermal_output(step, time, temperature) for a ThermalPhysics;
    write_pvd() at the end (the reference's destructor writes it)."""

    def __init__(self, physics, filename_prefix: str, output_dir: str = ""):
        self.physics = physics
        self.prefix = filename_prefix
        self.output_dir = output_dir
        self._times: List[Tuple[float, str]] = []

    def write_thermal_output(self, time_step: int, time: float, temperature, active=None):
        """temperature: the handle's device vector; active: the cells with
        material (default: the handle's, activations included)."""
        phys = self.physics
        cfg = phys.config
        geo = cfg.geometry
        grid = phys.to_grid(temperature)
        if active is None:
            active = phys.active_cells()
        phys.set_state_to_material_properties()
        state = phys.get_cell_state()
        piece = f"{self.prefix}.{time_step}.0.vtu"
        write_vtu(os.path.join(self.output_dir, piece), time, geo.n_cells, geo.extent, geo.origin, cfg.degree, grid,
                  active, state)
        record = f"{self.prefix}.{time_step}.pvtu"
        write_pvtu_record(os.path.join(self.output_dir, record), [piece])
        self._times.append((float(time), os.path.join(self.output_dir, record)))

    def write_pvd(self):
        write_pvd(os.path.join(self.output_dir, self.prefix + ".pvd"), self._times)
