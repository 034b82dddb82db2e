"""Problem description for the thermal hot path, mirroring adamantine's input database.

The reference reads a Boost property tree (``.info``/``.json``); the keys used
here are the ones that reach the thermal operator:

* geometry: ``length``/``width``/``height`` and their ``*_divisions`` and
  ``*_origin``, ``material_height``, ``use_powder``, ``powder_layer``
  (source/Geometry.cc:186-262, :317-353),
* materials: ``property_format``, ``n_materials``,
  ``material_X.<state>.<property>`` and the state-independent
  ``material_X.<property>`` (source/MaterialProperty.templates.hh:796-1119),
* boundary: ``type``, ``boundary_N.type``, ``printed_surface.type``
  (source/Boundary.cc:12-70),
* sources: ``beam_X.type`` goldak/electron_beam/cube with ``depth``,
  ``diameter``, ``max_power``, ``absorption_efficiency`` and a scan path
  (source/BeamHeatSourceProperties.hh:55-66, source/ScanPath.cc:58-195,
  source/CubeHeatSource.cc:14-43),
* time_stepping: ``method`` forward_euler / rk_third_order /
  rk_fourth_order (source/ThermalPhysics.templates.hh:449-471), plus
  ``rk_second_order`` (explicit midpoint, no counterpart in the reference).

Everything is plain Python/numpy: the module builds the ``adm_config`` C
structure declared in ``include/adamantine_b200.h``.
"""
from __future__ import annotations

import ctypes
import math
import sys
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

MAX_MATERIALS = 4
N_STATE_PROPERTIES = 8
MAX_STATES = 3
MAX_POLY = 5
TABLE_SIZE = 12
N_PROPERTIES = 5
MAX_SOURCES = 4
MAX_BOUNDARY_TYPES = 8
DBL_MAX = sys.float_info.max

STATE_NAMES = ("solid", "liquid", "powder")  # source/types.hh:107-108
STATE_PROPERTY_NAMES = (  # source/types.hh:40-49 (thermal ones)
    "density",
    "specific_heat",
    "thermal_conductivity_x",
    "thermal_conductivity_y",
    "thermal_conductivity_z",
    "emissivity",
    "radiation_heat_transfer_coef",
    "convection_heat_transfer_coef",
)
PROPERTY_NAMES = (  # source/types.hh:88-96
    "liquidus",
    "solidus",
    "latent_heat",
    "radiation_temperature_infty",
    "convection_temperature_infty",
)
BOUNDARY_BITS = {  # source/Boundary.hh enum BoundaryType
    "adiabatic": 0x1,
    "radiative": 0x2,
    "convective": 0x4,
    "clamped": 0x8,
    "traction_free": 0x10,
}
TIME_METHODS = {
    "forward_euler": 0,
    "rk_second_order": 1,
    "rk_third_order": 2,
    "rk_fourth_order": 3,
}
SOURCE_TYPES = {"goldak": 0, "electron_beam": 1, "cube": 2}
N_STAGES = {0: 1, 1: 2, 2: 3, 3: 4}


# --------------------------------------------------------------------------
# C structures (layout of adm_config in include/adamantine_b200.h)
# --------------------------------------------------------------------------
class SourceStruct(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int32),
        ("n_segments", ctypes.c_int32),
        ("depth", ctypes.c_double),
        ("absorption_efficiency", ctypes.c_double),
        ("radius_squared", ctypes.c_double),
        ("max_power", ctypes.c_double),
        ("cube_start_time", ctypes.c_double),
        ("cube_end_time", ctypes.c_double),
        ("cube_value", ctypes.c_double),
        ("cube_min", ctypes.c_double * 3),
        ("cube_max", ctypes.c_double * 3),
        ("segments", ctypes.POINTER(ctypes.c_double)),
    ]


class ConfigStruct(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32),
        ("degree", ctypes.c_int32),
        ("quadrature", ctypes.c_int32),
        ("n_cells", ctypes.c_int32 * 3),
        ("origin", ctypes.c_double * 3),
        ("extent", ctypes.c_double * 3),
        ("n_materials", ctypes.c_int32),
        ("n_states", ctypes.c_int32),
        ("use_table", ctypes.c_int32),
        ("p_order", ctypes.c_int32),
        ("poly", ctypes.c_double * (MAX_MATERIALS * N_STATE_PROPERTIES * MAX_STATES * MAX_POLY)),
        ("table", ctypes.c_double * (MAX_MATERIALS * N_STATE_PROPERTIES * MAX_STATES * TABLE_SIZE * 2)),
        ("props", ctypes.c_double * (MAX_MATERIALS * N_PROPERTIES)),
        ("n_boundary_types", ctypes.c_int32),
        ("boundary_types", ctypes.c_int32 * MAX_BOUNDARY_TYPES),
        ("n_sources", ctypes.c_int32),
        ("pad0", ctypes.c_int32),
        ("sources", SourceStruct * MAX_SOURCES),
        ("time_method", ctypes.c_int32),
        ("n_threads", ctypes.c_int32),
    ]


# --------------------------------------------------------------------------
# Geometry
# --------------------------------------------------------------------------
@dataclass
class Geometry:
    """Structured box (GridGenerator::subdivided_hyper_rectangle, colorize=true).

    Axis convention of source/Geometry.cc:188-253: in 3D coordinate 0 is the
    length (x), 1 the width (y) and 2 the height (z); in 2D coordinate 1 is
    the height.  ``n_cells`` and ``extent`` follow the same order.
    """

    dim: int
    n_cells: Sequence[int]
    extent: Sequence[float]
    origin: Sequence[float] = (0.0, 0.0, 0.0)
    material_height: float = 1e9
    use_powder: bool = False
    powder_layer: float = 0.0

    @property
    def n_cells_total(self) -> int:
        return int(np.prod(self.n_cells[: self.dim]))

    def cell_centers_height(self) -> np.ndarray:
        """Height coordinate of every cell centre (lexicographic, x fastest)."""
        zax = self.dim - 1
        nz = self.n_cells[zax]
        h = self.extent[zax] / nz
        zc = self.origin[zax] + (np.arange(nz) + 0.5) * h
        shape = tuple(reversed(self.n_cells[: self.dim]))
        out = np.broadcast_to(zc.reshape((nz,) + (1,) * (self.dim - 1)), shape)
        return np.ascontiguousarray(out).reshape(-1)

    def active_cells(self) -> np.ndarray:
        """FE_Q cells: centre below material_height (ThermalPhysics.templates.hh:472-493)."""
        return (self.cell_centers_height() < self.material_height).astype(np.uint8)

    def initial_state(self) -> np.ndarray:
        """Geometry::assign_material_state (source/Geometry.cc:317-353)."""
        zc = self.cell_centers_height()
        if self.use_powder:
            solid_height = self.material_height - self.powder_layer
            return np.where(zc < solid_height, 0, 2).astype(np.uint8)
        return np.zeros(zc.shape, np.uint8)

    def n_nodes(self, degree: int) -> int:
        return int(np.prod([degree * n + 1 for n in self.n_cells[: self.dim]]))

    def node_shape(self, degree: int):
        return tuple(degree * n + 1 for n in self.n_cells[: self.dim])


# --------------------------------------------------------------------------
# Material
# --------------------------------------------------------------------------
@dataclass
class Material:
    """Material tables of MaterialProperty (source/MaterialProperty.hh:359-383)."""

    n_states: int = 1
    n_materials: int = 1
    use_table: bool = False
    p_order: int = 0
    poly: np.ndarray = field(
        default_factory=lambda: np.zeros((MAX_MATERIALS, N_STATE_PROPERTIES, MAX_STATES, MAX_POLY))
    )
    table: np.ndarray = field(
        default_factory=lambda: np.zeros((MAX_MATERIALS, N_STATE_PROPERTIES, MAX_STATES, TABLE_SIZE, 2))
    )
    props: np.ndarray = field(default_factory=lambda: np.full((MAX_MATERIALS, N_PROPERTIES), DBL_MAX))

    @classmethod
    def from_database(cls, db: Dict[str, object], n_states: int, p_order: Optional[int] = None) -> "Material":
        """Parse ``materials`` keys as MaterialProperty::fill_properties does
        (source/MaterialProperty.templates.hh:796-1119)."""
        fmt = str(db.get("property_format", "polynomial"))
        n_mat = int(db.get("n_materials", 1))
        if n_mat > MAX_MATERIALS:
            raise ValueError(f"at most {MAX_MATERIALS} materials are supported")
        m = cls(n_states=n_states, n_materials=n_mat, use_table=(fmt == "table"))
        max_len = 1
        for mat in range(n_mat):
            for s in range(n_states):
                for p, pname in enumerate(STATE_PROPERTY_NAMES):
                    key = f"material_{mat}.{STATE_NAMES[s]}.{pname}"
                    if key not in db:
                        continue
                    text = "".join(str(db[key]).split())
                    if m.use_table:
                        pairs = [x for x in text.split("|") if x]
                        if len(pairs) > TABLE_SIZE:
                            raise ValueError("Too many coefficients, increase the table size")
                        for i, pair in enumerate(pairs):
                            t, v = pair.split(",")
                            m.table[mat, p, s, i] = (float(t), float(v))
                        for i in range(len(pairs), TABLE_SIZE):
                            m.table[mat, p, s, i] = m.table[mat, p, s, i - 1]
                    else:
                        coefs = [float(x) for x in text.split(",") if x != ""]
                        if len(coefs) > MAX_POLY:
                            raise ValueError("Too many coefficients, increase the polynomial order")
                        max_len = max(max_len, len(coefs))
                        m.poly[mat, p, s, : len(coefs)] = coefs
            for p, pname in enumerate(PROPERTY_NAMES):
                key = f"material_{mat}.{pname}"
                m.props[mat, p] = float(db[key]) if key in db else DBL_MAX
        m.p_order = (max_len - 1) if p_order is None else int(p_order)
        if not m.use_table and max_len - 1 > m.p_order:
            raise ValueError("Too many coefficients, increase the polynomial order")
        return m


# --------------------------------------------------------------------------
# Boundary
# --------------------------------------------------------------------------
def parse_boundary_line(text: str) -> int:
    """Boundary::parse_boundary_line (source/Boundary.cc:87-109)."""
    bits = 0
    for tok in str(text).split(","):
        bits |= BOUNDARY_BITS[tok.strip()]
    return bits


@dataclass
class Boundary:
    types: List[int]

    @classmethod
    def from_database(cls, db: Dict[str, str], dim: int) -> "Boundary":
        """Boundary ctor (source/Boundary.cc:12-70) for the 2*dim colorized ids."""
        n = 2 * dim
        default = parse_boundary_line(db["type"]) if "type" in db else 0
        types = [default] * n
        for i in range(n):
            key = f"boundary_{i}.type"
            if key in db:
                types[i] = parse_boundary_line(db[key])
        if "printed_surface.type" in db:
            types[-1] = parse_boundary_line(db["printed_surface.type"])
        return cls(types)

    @property
    def adiabatic_only(self) -> bool:
        return all(t & BOUNDARY_BITS["adiabatic"] for t in self.types)


# --------------------------------------------------------------------------
# Sources and scan paths
# --------------------------------------------------------------------------
def parse_scan_path(text: str, file_format: str = "segment", distance_scaling: float = 1.0,
                    velocity_scaling: float = 1.0) -> np.ndarray:
    """ScanPath::load_segment_scan_path / load_event_series_scan_path
    (source/ScanPath.cc:58-195).  Returns an (n, 5) array of
    (end_time, power_modifier, x, y, z).  Five-axis rotations are not kept."""
    rows: List[List[float]] = []
    lines = text.splitlines()
    if file_format == "segment":
        n_segments = int(lines[1])
        for line in lines[3:]:
            if len(rows) >= n_segments:
                break
            if "SCAN_PATH_END" in line:
                break
            tok = line.split()
            if not tok:
                continue
            end = [float(tok[1]) * distance_scaling, float(tok[2]) * distance_scaling,
                   float(tok[3]) * distance_scaling]
            pmod = float(tok[4])
            if tok[0] == "1":
                end_time = (rows[-1][0] if rows else 0.0) + float(tok[5])
            elif tok[0] == "0":
                if not rows:
                    raise ValueError("Error: Scan paths must begin with a 'point' segment.")
                velocity = float(tok[5]) * velocity_scaling
                prev = rows[-1][2:5]
                length = math.sqrt(sum((a - b) ** 2 for a, b in zip(end, prev)))
                end_time = rows[-1][0] + abs(length / velocity)
            else:
                raise ValueError("scan path mode not recognized")
            rows.append([end_time, pmod] + end)
    elif file_format == "event_series":
        last_power = 0.0
        for line in lines:
            if line == "":
                continue
            if "SCAN_PATH_END" in line:
                break
            tok = [t for t in line.replace(",", " ").split() if t]
            rows.append([float(tok[0]), last_power, float(tok[1]) * distance_scaling,
                         float(tok[2]) * distance_scaling, float(tok[3]) * distance_scaling])
            last_power = float(tok[-1])
    else:
        raise ValueError("Error: Format of scan path file not recognized.")
    return np.asarray(rows, dtype=np.float64).reshape(-1, 5)


@dataclass
class Source:
    type: str = "goldak"
    depth: float = 0.0
    absorption_efficiency: float = 0.0
    diameter: float = 0.0
    max_power: float = 0.0
    segments: np.ndarray = field(default_factory=lambda: np.zeros((0, 5)))
    cube_start_time: float = 0.0
    cube_end_time: float = 0.0
    cube_value: float = 0.0
    cube_min: Sequence[float] = (0.0, 0.0, 0.0)
    cube_max: Sequence[float] = (0.0, 0.0, 0.0)

    @property
    def radius_squared(self) -> float:
        # BeamHeatSourceProperties::set_from_database: radius = diameter / 2
        return (self.diameter / 2.0) ** 2


@dataclass
class ThermalConfig:
    geometry: Geometry
    material: Material
    boundary: Boundary
    sources: List[Source] = field(default_factory=list)
    degree: int = 1
    quadrature: str = "gauss"
    time_method: str = "forward_euler"
    n_threads: int = 0

    @property
    def n_nodes(self) -> int:
        return self.geometry.n_nodes(self.degree)

    @property
    def n_cells(self) -> int:
        return self.geometry.n_cells_total

    @property
    def n_qp(self) -> int:
        return (self.degree + 1) ** self.geometry.dim

    @property
    def n_stages(self) -> int:
        return N_STAGES[TIME_METHODS[self.time_method]]

    def to_struct(self) -> ConfigStruct:
        """Fill the C structure. The returned object keeps the segment
        buffers alive (``_keep``)."""
        g, m = self.geometry, self.material
        c = ConfigStruct()
        c.dim = g.dim
        c.degree = self.degree
        c.quadrature = 1 if self.quadrature == "gauss_lobatto" else 0
        for d in range(3):
            c.n_cells[d] = int(g.n_cells[d]) if d < g.dim else 1
            c.origin[d] = float(g.origin[d]) if d < len(g.origin) else 0.0
            c.extent[d] = float(g.extent[d]) if d < g.dim else 1.0
        c.n_materials = m.n_materials
        c.n_states = m.n_states
        c.use_table = int(bool(m.use_table))
        c.p_order = m.p_order
        ctypes.memmove(c.poly, np.ascontiguousarray(m.poly, np.float64).ctypes.data, ctypes.sizeof(c.poly))
        ctypes.memmove(c.table, np.ascontiguousarray(m.table, np.float64).ctypes.data, ctypes.sizeof(c.table))
        ctypes.memmove(c.props, np.ascontiguousarray(m.props, np.float64).ctypes.data, ctypes.sizeof(c.props))
        if len(self.boundary.types) > MAX_BOUNDARY_TYPES:
            raise ValueError("too many boundary types")
        c.n_boundary_types = len(self.boundary.types)
        for i, t in enumerate(self.boundary.types):
            c.boundary_types[i] = int(t)
        if len(self.sources) > MAX_SOURCES:
            raise ValueError(f"at most {MAX_SOURCES} heat sources are supported")
        c.n_sources = len(self.sources)
        keep = []
        for i, s in enumerate(self.sources):
            ss = c.sources[i]
            ss.type = SOURCE_TYPES[s.type]
            seg = np.ascontiguousarray(s.segments, np.float64).reshape(-1, 5)
            keep.append(seg)
            ss.n_segments = seg.shape[0]
            ss.segments = seg.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if seg.size else None
            ss.depth = s.depth
            ss.absorption_efficiency = s.absorption_efficiency
            ss.radius_squared = s.radius_squared
            ss.max_power = s.max_power
            ss.cube_start_time = s.cube_start_time
            ss.cube_end_time = s.cube_end_time
            ss.cube_value = s.cube_value
            for d in range(3):
                ss.cube_min[d] = s.cube_min[d] if d < len(s.cube_min) else 0.0
                ss.cube_max[d] = s.cube_max[d] if d < len(s.cube_max) else 0.0
        c.time_method = TIME_METHODS[self.time_method]
        c.n_threads = int(self.n_threads)
        c._keep = keep  # type: ignore[attr-defined]
        return c
