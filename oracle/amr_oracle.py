"""Refined-mesh restatement of the thermal path -- TEST INFRASTRUCTURE ONLY
(tests/ import it as the checker; nothing in the package uses it).

Follows the reference's adaptive path:
  * compute_cells_to_refine (application/adamantine.hh:540-606) with
    HeatSource::get_bounding_box (GoldakHeatSource.cc:152-190,
    ElectronBeamHeatSource.cc:162-200, CubeHeatSource.cc:111-123) and
    ScanPath::value (ScanPath.cc:228-257);
  * refine_mesh (application/adamantine.hh:608-681): n_refinements rounds of
    coarsen / refine flags and an execution;
  * hanging-node constraints (make_hanging_node_constraints,
    application/adamantine.hh:514-523) on meshes balanced 2:1 across faces
    and edges;
  * the constrained operator (ThermalOperator.templates.hh:205-224) and the
    inverse mass (:140-160), each level's cells applied by the CPU oracle of
    the uniform path (oracle_py.Oracle) on that level's grid;
  * refine_and_transfer (application/adamantine.hh:312-539): the old field
    evaluated at the new nodes, cell states copied to children / taken from
    first children.

Written independently of the package's implementation: node positions are
floating-point coordinates (so Gauss-Lobatto nodes of any degree work),
hanging nodes are found by locating each node in the coarser active leaves
that contain it, and constraint weights are the coarse cell's full
tensor-product basis evaluated there.

Assumptions where the reference's behaviour lives in deal.II / p4est (not in
the reference tree): balance is 2:1 across faces and edges, coarsening that
would break it is skipped, families are coarsened level by level from the
finest, parents in lexicographic order, and coarsening takes the first
child's cell data.
"""
from __future__ import annotations

import copy
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from oracle_py import Oracle

SCALE = float(1 << 24)  # key resolution per coarse cell


def gl_nodes(p: int) -> List[float]:
    """Gauss-Lobatto points on [0, 1] (FE_Q support points)."""
    if p == 1:
        return [0.0, 1.0]
    if p == 2:
        return [0.0, 0.5, 1.0]
    if p == 3:
        s = 1.0 / math.sqrt(5.0)
        return [0.0, 0.5 * (1 - s), 0.5 * (1 + s), 1.0]
    if p == 4:
        s = math.sqrt(3.0 / 7.0)
        return [0.0, 0.5 * (1 - s), 0.5, 0.5 * (1 + s), 1.0]
    raise ValueError("degree 1..4")


def lagrange(nodes: Sequence[float], a: int, u: float) -> float:
    v = 1.0
    for b, xb in enumerate(nodes):
        if b != a:
            v *= (u - xb) / (nodes[a] - xb)
    return v


FACE_EDGE = [(x, y, z) for z in (-1, 0, 1) for y in (-1, 0, 1) for x in (-1, 0, 1)
             if 1 <= (x != 0) + (y != 0) + (z != 0) <= 2]


def tableau(method: int):
    """deal.II ExplicitRungeKutta tableaux (ThermalPhysics.templates.hh:449-471)."""
    if method == 0:
        return [[]], [1.0], [0.0]
    if method == 1:
        return [[], [0.5]], [0.0, 1.0], [0.0, 0.5]
    if method == 2:
        return [[], [0.5], [-1.0, 2.0]], [1 / 6, 2 / 3, 1 / 6], [0.0, 0.5, 1.0]
    return [[], [0.5], [0.0, 0.5], [0.0, 0.0, 1.0]], [1 / 6, 1 / 3, 1 / 3, 1 / 6], [0.0, 0.5, 0.5, 1.0]


class Forest:
    """Leaves (level, i, j, k) of a forest of octrees over nc coarse cells."""

    def __init__(self, nc, max_level: int):
        self.nc = tuple(int(n) for n in nc)
        self.L = int(max_level)
        self.leaves = {(0, i, j, k) for k in range(self.nc[2]) for j in range(self.nc[1]) for i in range(self.nc[0])}

    def n(self, l, d):
        return self.nc[d] << l

    def inside(self, l, c):
        return all(0 <= c[d] < self.n(l, d) for d in range(3))

    def find(self, l, c):
        """The leaf whose region holds cell (l, c); None when that cell is refined."""
        for m in range(l, -1, -1):
            s = l - m
            key = (m, c[0] >> s, c[1] >> s, c[2] >> s)
            if key in self.leaves:
                return key
        return None

    @staticmethod
    def children(cell):
        l, i, j, k = cell
        return [(l + 1, 2 * i + (q & 1), 2 * j + ((q >> 1) & 1), 2 * k + (q >> 2)) for q in range(8)]

    def refine(self, cell):
        self.leaves.remove(cell)
        self.leaves.update(self.children(cell))

    def coarsen(self, parent):
        for c in self.children(parent):
            self.leaves.remove(c)
        self.leaves.add(parent)

    def balance(self):
        changed = True
        while changed:
            changed = False
            for leaf in sorted(self.leaves):
                if leaf not in self.leaves:
                    continue
                l = leaf[0]
                for o in FACE_EDGE:
                    nb = (leaf[1] + o[0], leaf[2] + o[1], leaf[3] + o[2])
                    if not self.inside(l, nb):
                        continue
                    f = self.find(l, nb)
                    if f is not None and f[0] < l - 1:
                        self.refine(f)
                        changed = True

    def keeps_balance(self, parent):
        l = parent[0]
        for ch in self.children(parent):
            for o in FACE_EDGE:
                nb = (ch[1] + o[0], ch[2] + o[1], ch[3] + o[2])
                if not self.inside(l + 1, nb) or (nb[0] >> 1, nb[1] >> 1, nb[2] >> 1) == parent[1:]:
                    continue
                if self.find(l + 1, nb) is None:
                    return False
        return True

    def execute(self, refine: set, coarsen: set):
        old = set(self.leaves)
        for cell in sorted(refine, key=lambda c: (c[0], c[3], c[2], c[1])):
            if cell in old and cell[0] < self.L:
                self.refine(cell)
        for l in range(self.L - 1, -1, -1):
            for k in range(self.n(l, 2)):
                for j in range(self.n(l, 1)):
                    for i in range(self.n(l, 0)):
                        par = (l, i, j, k)
                        if par in self.leaves:
                            continue
                        ch = self.children(par)
                        if all(c in self.leaves and c in old and c in coarsen for c in ch) and self.keeps_balance(par):
                            self.coarsen(par)
        self.balance()

    def sorted_leaves(self):
        return sorted(self.leaves, key=lambda c: (c[0], c[3], c[2], c[1]))


def beam_center(segments: np.ndarray, t: float):
    """ScanPath::value: linear between segment end points (rows: end_time,
    power_modifier, x, y, z); after the last one a point far outside."""
    seg = np.asarray(segments, np.float64).reshape(-1, 5)
    n = len(seg)
    if n == 0 or t > seg[-1, 0]:
        low = -np.finfo(np.float64).max
        return np.array([low, low, low])
    cur = int(np.searchsorted(seg[:, 0], t, side="left"))
    start_t = seg[cur - 1, 0] if cur > 0 else 0.0
    start_p = seg[cur - 1, 2:5] if cur > 0 else seg[cur, 2:5]
    return start_p + (seg[cur, 2:5] - start_p) / (seg[cur, 0] - start_t) * (t - start_t)


class AmrProblem:
    """The refined thermal problem: cfg a ThermalConfig (its geometry is the
    coarse mesh), coarse-cell active / material / initial-state arrays."""

    def __init__(self, cfg, max_level: int, active=None, material_id=None, initial_state=None):
        self.cfg = cfg
        g = cfg.geometry
        self.nc = tuple(int(n) for n in g.n_cells)
        self.p = int(cfg.degree)
        self.gl = gl_nodes(self.p)
        self.forest = Forest(self.nc, max_level)
        C = int(np.prod(self.nc))
        self.coarse_active = np.ones(C, np.uint8) if active is None else np.asarray(active, np.uint8).reshape(C)
        self.coarse_mat = np.zeros(C, np.uint8) if material_id is None else np.asarray(material_id, np.uint8).reshape(C)
        self.coarse_init = (np.zeros(C, np.uint8) if initial_state is None
                            else np.asarray(initial_state, np.uint8).reshape(C))
        self.y = None
        self.levels: Dict[int, dict] = {}

    # ------------------------------------------------------------ mesh
    def coarse_index(self, l, c):
        s = l
        return (c[0] >> s) + self.nc[0] * ((c[1] >> s) + self.nc[1] * (c[2] >> s))

    def active_leaf(self, cell):
        return cell in self.forest.leaves and self.coarse_active[self.coarse_index(cell[0], cell[1:])] != 0

    def cells_to_refine(self, time, next_time, n_steps):
        boxes = []
        for s in range(n_steps):
            t = time + s / n_steps * (next_time - time)
            for src in self.cfg.sources:
                if src.type == "cube":
                    boxes.append((np.asarray(src.cube_min, float), np.asarray(src.cube_max, float)))
                    continue
                c = beam_center(src.segments, t)
                r = math.sqrt(src.radius_squared)
                lo = np.array([c[0] - 2 * r, c[1] - 2 * r, c[2] - 2 * src.depth])
                hi = np.array([c[0] + 2 * r, c[1] + 2 * r, c[2]])
                boxes.append((lo, hi))
        g = self.cfg.geometry
        out = set()
        for cell in self.forest.leaves:
            l = cell[0]
            h = [g.extent[d] / self.forest.n(l, d) for d in range(3)]
            lo = [g.origin[d] + cell[1 + d] * h[d] for d in range(3)]
            hi = [g.origin[d] + (cell[1 + d] + 1) * h[d] for d in range(3)]
            for blo, bhi in boxes:
                if all(lo[d] <= bhi[d] and blo[d] <= hi[d] for d in range(3)):
                    out.add(cell)
                    break
        return out

    def refine_mesh_flags(self, time, next_time, n_steps, n_refinements, coarsen_after_beam):
        """One application of refine_mesh's rounds to the forest."""
        for _ in range(n_refinements):
            hit = self.cells_to_refine(time, next_time, n_steps)
            coarsen = {c for c in self.forest.leaves if coarsen_after_beam and c[0] > 0 and c not in hit}
            refine = {c for c in hit if c[0] < n_refinements}
            self.forest.execute(refine, coarsen)

    def node_positions(self, cell):
        """(a, b, c, x) of the cell's nodes, x in coarse-cell units."""
        l, i, j, k = cell
        f = 1.0 / (1 << l)
        out = []
        for c in range(self.p + 1):
            for b in range(self.p + 1):
                for a in range(self.p + 1):
                    x = ((i + self.gl[a]) * f, (j + self.gl[b]) * f, (k + self.gl[c]) * f)
                    out.append((a, b, c, x))
        return out

    @staticmethod
    def key(x):
        return tuple(int(round(v * SCALE)) for v in x)

    def locate(self, x, max_level):
        """Active leaves of level < max_level whose closed box holds x."""
        for m in range(max_level):
            cand = []
            for d in range(3):
                v = x[d] * (1 << m)
                f = math.floor(v + 1e-12)
                opts = [f]
                if abs(v - round(v)) < 1e-12:
                    opts = [int(round(v)) - 1, int(round(v))]
                cand.append([o for o in opts if 0 <= o < self.forest.n(m, d)])
            for c in cand[2]:
                for b in cand[1]:
                    for a in cand[0]:
                        cell = (m, a, b, c)
                        if self.active_leaf(cell):
                            yield cell

    def build(self):
        """DoFs (non-hanging nodes, sorted by z, y, x) and constraints."""
        pos: Dict[tuple, tuple] = {}
        owner_level: Dict[tuple, int] = {}
        for cell in self.forest.leaves:
            if not self.active_leaf(cell):
                continue
            for a, b, c, x in self.node_positions(cell):
                k = self.key(x)
                pos[k] = x
                owner_level[k] = max(owner_level.get(k, 0), cell[0])
        hang: Dict[tuple, List[Tuple[tuple, float]]] = {}
        for k, x in pos.items():
            for C in self.locate(x, owner_level[k]):
                m = C[0]
                u = [x[d] * (1 << m) - C[1 + d] for d in range(3)]
                if all(any(abs(ud - g) < 1e-12 for g in self.gl) for ud in u):
                    continue  # a node of C
                ent = []
                for c in range(self.p + 1):
                    for b in range(self.p + 1):
                        for a in range(self.p + 1):
                            w = lagrange(self.gl, a, u[0]) * lagrange(self.gl, b, u[1]) * lagrange(self.gl, c, u[2])
                            if abs(w) > 1e-14:
                                xm = ((C[1] + self.gl[a]) / (1 << m), (C[2] + self.gl[b]) / (1 << m),
                                      (C[3] + self.gl[c]) / (1 << m))
                                ent.append((self.key(xm), w))
                hang[k] = ent
                break
        # resolve constraints whose masters hang themselves
        resolved = {}
        for k, ent in hang.items():
            cur = ent
            for _ in range(8):
                nxt, again = [], False
                for mk, w in cur:
                    if mk in hang:
                        again = True
                        nxt.extend((mk2, w * w2) for mk2, w2 in hang[mk])
                    else:
                        nxt.append((mk, w))
                cur = nxt
                if not again:
                    break
            acc: Dict[tuple, float] = {}
            for mk, w in cur:
                acc[mk] = acc.get(mk, 0.0) + w
            resolved[k] = acc
        self.dof_keys = sorted((k for k in pos if k not in hang), key=lambda k: (k[2], k[1], k[0]))
        self.dof_of = {k: d for d, k in enumerate(self.dof_keys)}
        self.hanging = {k: {self.dof_of[mk]: w for mk, w in v.items()} for k, v in resolved.items()}
        self.positions = pos
        self.n_dofs = len(self.dof_keys)

    def dof_points(self):
        return np.array([self.positions[k] for k in self.dof_keys])

    def entries(self, k):
        if k in self.dof_of:
            return {self.dof_of[k]: 1.0}
        return self.hanging[k]

    # ------------------------------------------------------- level grids
    def level_config(self, l):
        cfg = copy.deepcopy(self.cfg)
        cfg.geometry.n_cells = tuple(n << l for n in self.nc)
        return cfg

    def setup_levels(self, states=None):
        """Level oracles; states: per level cell-state arrays (None: the
        coarse cells' initial states)."""
        self.levels = {}
        p = self.p
        for l in range(self.forest.L + 1):
            cells = [c for c in self.forest.leaves if c[0] == l and self.active_leaf(c)]
            if not cells:
                continue
            n = [self.forest.n(l, d) for d in range(3)]
            C = n[0] * n[1] * n[2]
            act = np.zeros(C, np.uint8)
            dom = np.zeros(C, np.uint8)
            mat = np.zeros(C, np.uint8)
            init = np.zeros(C, np.uint8)
            for k in range(n[2]):
                for j in range(n[1]):
                    for i in range(n[0]):
                        idx = i + n[0] * (j + n[1] * k)
                        ci = self.coarse_index(l, (i, j, k))
                        dom[idx] = self.coarse_active[ci]
                        mat[idx] = self.coarse_mat[ci]
                        init[idx] = self.coarse_init[ci]
            for c in cells:
                act[c[1] + n[0] * (c[2] + n[1] * c[3])] = 1
            cfg = self.level_config(l)
            st = cfg.to_struct()
            orc = Oracle(st, active=act, material_id=mat, initial_state=init, domain=dom)
            orc._keep = st
            if states is not None and l in states:
                orc.set_cell_state(states[l])
                orc.get_state_from_material_properties()
            nn = [p * n[d] + 1 for d in range(3)]
            rows: Dict[int, dict] = {}
            for cell in cells:
                for a, b, c, x in self.node_positions(cell):
                    node = (p * cell[1] + a) + nn[0] * ((p * cell[2] + b) + nn[1] * (p * cell[3] + c))
                    if node not in rows:
                        rows[node] = self.entries(self.key(x))
            self.levels[l] = {"oracle": orc, "n": n, "nn": nn, "rows": rows, "cells": cells}
        self.compute_inverse_mass()

    def prolong(self, y, l):
        lev = self.levels[l]
        out = np.zeros(lev["oracle"].n_nodes)
        for node, ent in lev["rows"].items():
            out[node] = sum(w * y[d] for d, w in ent.items())
        return out

    def restrict(self, per_level):
        out = np.zeros(self.n_dofs)
        for l, vec in per_level.items():
            for node, ent in self.levels[l]["rows"].items():
                for d, w in ent.items():
                    out[d] += w * vec[node]
        return out

    def compute_inverse_mass(self):
        per = {}
        for l, lev in self.levels.items():
            im = lev["oracle"].inverse_mass()
            m = np.zeros_like(im)
            nz = im > 0
            m[nz] = 1.0 / im[nz]
            per[l] = m
        mass = self.restrict(per)
        self.inv_mass = np.where(mass > 0, 1.0 / np.where(mass > 0, mass, 1.0), 0.0)

    def set_time(self, t):
        for lev in self.levels.values():
            lev["oracle"].set_time(t)

    def vmult(self, src):
        per = {l: lev["oracle"].vmult(self.prolong(src, l)) for l, lev in self.levels.items()}
        return self.restrict(per)

    def setup(self, initial_temperature: float):
        self.build()
        self.setup_levels()
        self.y = np.full(self.n_dofs, float(initial_temperature))

    def evolve_one_time_step(self, t, dt):
        a, b, c = tableau(self.cfg.to_struct().time_method)
        ks = []
        for i in range(len(b)):
            z = self.y.copy()
            for j, aij in enumerate(a[i]):
                if aij != 0.0:
                    z = z + dt * aij * ks[j]
            self.set_time(t + c[i] * dt)
            ks.append(self.inv_mass * self.vmult(z))
        for i, bi in enumerate(b):
            if bi != 0.0:
                self.y = self.y + dt * bi * ks[i]
        return t + dt

    # ------------------------------------------------------- transfer
    def evaluate(self, x, level_values):
        """The field at x from the active leaf that holds it."""
        for cell in self.locate(x, self.forest.L + 1):
            l = cell[0]
            lev = self.levels[l]
            nn = lev["nn"]
            u = [x[d] * (1 << l) - cell[1 + d] for d in range(3)]
            v = 0.0
            for c in range(self.p + 1):
                for b in range(self.p + 1):
                    for a in range(self.p + 1):
                        w = lagrange(self.gl, a, u[0]) * lagrange(self.gl, b, u[1]) * lagrange(self.gl, c, u[2])
                        node = (self.p * cell[1] + a) + nn[0] * ((self.p * cell[2] + b) + nn[1] * (self.p * cell[3] + c))
                        v += w * level_values[l][node]
            return v
        raise RuntimeError("point outside the material")

    def remesh(self, change):
        """refine_and_transfer around change(forest)."""
        old_forest = copy.deepcopy(self.forest)
        old_levels = self.levels
        vals = {l: self.prolong(self.y, l) for l in old_levels}
        ns = int(self.cfg.to_struct().n_states)
        states = {}
        for l, lev in old_levels.items():
            lev["oracle"].set_state_to_material_properties()
            states[l] = np.asarray(lev["oracle"].cell_state()).reshape(ns, -1)
        change(self.forest)
        new_forest = self.forest
        self.build()
        # new cell states: the old leaf holding the new leaf, or its first child
        new_states = {}
        for l in range(new_forest.L + 1):
            cells = [c for c in new_forest.leaves if c[0] == l and self.active_leaf(c)]
            if not cells:
                continue
            n = [new_forest.n(l, d) for d in range(3)]
            st = np.zeros((ns, n[0] * n[1] * n[2]))
            for cell in cells:
                src = old_forest.find(l, cell[1:])
                if src is None:
                    src = cell
                    while src not in old_forest.leaves:
                        src = old_forest.children(src)[0]
                m = src[0]
                nm = [old_forest.n(m, d) for d in range(3)]
                st[:, cell[1] + n[0] * (cell[2] + n[1] * cell[3])] = states[m][:, src[1] + nm[0] * (src[2] + nm[1] * src[3])]
            new_states[l] = st.reshape(-1)
        # the old field at the new nodes, located on the old mesh
        keys, positions = self.dof_keys, self.positions
        self.forest, self.levels = old_forest, old_levels
        y_new = np.array([self.evaluate(positions[k], vals) for k in keys])
        self.forest = new_forest
        self.setup_levels(new_states)
        self.y = y_new

    def refine_mesh(self, time, next_time, n_steps, n_refinements, coarsen_after_beam=False):
        self.remesh(lambda f: self.refine_mesh_flags(time, next_time, n_steps, n_refinements, coarsen_after_beam))

    def execute(self, refine: set, coarsen: set):
        self.remesh(lambda f: f.execute(refine, coarsen))

    def level_values(self, l):
        return self.prolong(self.y, l)
