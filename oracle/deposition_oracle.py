"""numpy restatement of the reference's material deposition -- test
infrastructure only (the checker of the library's box generation and of the
device activation), never part of the product path.

boxes_along_path follows deposition_along_scan_path
(source/material_deposition.cc:129-275) for three-axis scan paths, with the
same sequence of floating-point operations; cells_in_box follows
get_elements_to_activate (:374-438): a cell is selected when its closed
bounding box [x_i, x_{i+1}] x ... (vertices p1 + i * (p2 - p1) / n of a
subdivided hyper-rectangle) intersects the closed box.
"""
from __future__ import annotations

import math

import numpy as np


def boxes_along_path(seg, length, height, width, lead_time):
    eps, eps_time = 1.0e-10, 1.0e-10
    out = []
    start_time = 0.0
    start = [float(seg[0][2]), float(seg[0][3]), float(seg[0][4])]
    for row in seg:
        end = [float(row[2]), float(row[3]), float(row[4])]
        if row[1] > eps:
            L = math.sqrt((end[0] - start[0]) ** 2 + (end[1] - start[1]) ** 2 + (end[2] - start[2]) ** 2)
            center = list(start)
            v = L / (row[0] - start_time)
            c = (end[0] - start[0]) / L if L != 0.0 else 1.0
            s = (end[1] - start[1]) / L if L != 0.0 else 0.0
            blen = length
            while True:
                d = math.sqrt((center[0] - start[0]) ** 2 + (center[1] - start[1]) ** 2 +
                              (center[2] - start[2]) ** 2)
                tc = d / v if v != 0.0 else 0.0
                sx = abs(c) * blen + abs(s) * width
                sy = abs(c) * width + abs(s) * blen
                out.append([center[0] - 0.5 * sx, center[1] - 0.5 * sy, center[2] - height,
                            center[0] + 0.5 * sx, center[1] + 0.5 * sy, center[2],
                            max(start_time + tc - lead_time, eps_time), c, s])
                if d + eps > L:
                    break
                inc = length
                if d + length > L:
                    inc = L - d
                    blen = L - d
                center[0] += c * inc
                center[1] += s * inc
        start = end
        start_time = float(row[0])
    return np.array(out).reshape(-1, 9)


def cells_in_box(lo, hi, origin, h, n_cells):
    """Lexicographic indices (x fastest) of the cells meeting the box."""
    sel = []
    for d in range(3):
        i = np.arange(n_cells[d])
        x0 = origin[d] + i * h[d]
        x1 = origin[d] + (i + 1) * h[d]
        sel.append(i[(x0 <= hi[d]) & (x1 >= lo[d])])
    if any(s.size == 0 for s in sel):
        return np.zeros(0, np.int64)
    X, Y, Z = np.meshgrid(sel[0], sel[1], sel[2], indexing="ij")
    return np.sort((X + n_cells[0] * (Y + n_cells[1] * Z)).reshape(-1)).astype(np.int64)


def activate(active, lo, hi, b0, b1, origin, h, n_cells):
    """Cells newly activated by boxes [b0, b1) and the box that sets each
    one's direction (the last box meeting it)."""
    last = {}
    for b in range(b0, b1):
        for c in cells_in_box(lo[b], hi[b], origin, h, n_cells):
            if not active[c]:
                last[int(c)] = b
    cells = np.array(sorted(last), np.int64)
    return cells, np.array([last[c] for c in cells.tolist()], np.int64)
