"""numpy restatement of the reference's microstructure output -- test
infrastructure only (the checker of the GPU G/R kernel), never part of the
product path.

Microstructure::compute_G_and_R (source/Microstructure.hh:89-207): for every
active cell of a box mesh of FE_Q(p) elements, in the triangulation's cell
order, and every QGaussLobatto(p + 1) point of the cell (these are the
support points, lexicographic, x fastest), when the node there went from
above the cell's liquidus (old temperature) to at or below it (new
temperature), one record:
    the point's coordinates, G = |grad T| (T the new field, gradient of the
    cell's interpolant at the point), the cooling rate and R = rate / G,
where the cooling rate is computed as the reference writes it,
``_old_temperature[dof] - temperature[dof] / delta_t`` (:150): the division
binds to the new temperature only. A node shared by several cells gives one
record per cell, each with that cell's one-sided gradient. The lines are the
values separated by spaces with 9 significant digits (the reference's
std::setprecision(9)), "inf" where G is 0.
"""
from __future__ import annotations

import numpy as np


def nodal_derivative(degree):
    """D[a][i] = phi_i'(x_a) for the Lagrange basis on the points
    {0, 1/p, ..., 1} of [0, 1] (the Gauss-Lobatto points for p <= 2)."""
    x = np.linspace(0.0, 1.0, degree + 1)
    n = degree + 1
    D = np.zeros((n, n))
    for i in range(n):
        for a in range(n):
            # derivative of prod_{j != i} (x - x_j) / (x_i - x_j) at x_a
            s = 0.0
            for m in range(n):
                if m == i:
                    continue
                term = 1.0 / (x[i] - x[m])
                for j in range(n):
                    if j in (i, m):
                        continue
                    term *= (x[a] - x[j]) / (x[i] - x[j])
                s += term
            D[a, i] = s
    return D


def compute_G_and_R(n_cells, extent, degree, t_old, t_new, delta_t, liquidus, active=None, material=None,
                    origin=None):
    """n_cells, extent, origin: per axis (2 or 3 axes, x first). t_old,
    t_new: nodal grids of shape reversed(nodes) (slowest axis first), nodes =
    degree * n_cells + 1. liquidus: per material id. active, material: per
    cell (lexicographic, x fastest), default all active, material 0.
    Returns the records (n, dim + 3) in the reference's order."""
    dim = len(n_cells)
    origin = np.zeros(dim) if origin is None else np.asarray(origin, np.float64)
    h = np.asarray(extent, np.float64) / np.asarray(n_cells)
    n = degree + 1
    D = nodal_derivative(degree)
    pts = np.linspace(0.0, 1.0, n)
    To = np.asarray(t_old, np.float64)
    Tn = np.asarray(t_new, np.float64)
    n_total = int(np.prod(n_cells))
    act = np.ones(n_total, bool) if active is None else np.asarray(active) != 0
    mat = np.zeros(n_total, int) if material is None else np.asarray(material, int)
    liq = np.asarray(liquidus, np.float64)
    out = []
    for c in range(n_total):
        if not act[c]:
            continue
        cell = []
        r = c
        for d in range(dim):
            cell.append(r % n_cells[d])
            r //= n_cells[d]
        lq = liq[mat[c]]
        # the cell's nodal values, indexed [x][y](z)
        sl = tuple(slice(degree * cell[d], degree * cell[d] + n) for d in reversed(range(dim)))
        to = To[sl].transpose()
        tn = Tn[sl].transpose()
        cross = (to > lq) & (tn <= lq)
        if not cross.any():
            continue
        for q in np.ndindex(*([n] * dim)[::-1]):
            loc = q[::-1]  # (a, b[, k]), x fastest
            if not cross[loc]:
                continue
            grad = []
            for d in range(dim):
                line = [slice(None) if e == d else loc[e] for e in range(dim)]
                vals = tn[tuple(line)]
                s = 0.0
                for i in range(n):  # left to right, each product rounded
                    s = s + float(D[loc[d], i]) * float(vals[i])
                grad.append(s / h[d])
            G2 = 0.0
            for g in grad:
                G2 = G2 + g * g
            G = float(np.sqrt(G2))
            rate = float(to[loc]) - float(tn[loc]) / delta_t
            with np.errstate(divide="ignore", invalid="ignore"):
                R = np.float64(rate) / np.float64(G)
            x = [(origin[d] + cell[d] * h[d]) + pts[loc[d]] * h[d] for d in range(dim)]
            out.append(x + [G, rate, float(R)])
    return np.array(out, np.float64).reshape(-1, dim + 3)


def format_records(records):
    """The reference's text lines (std::setprecision(9), space separated)."""
    lines = []
    for r in np.asarray(records):
        lines.append(" ".join(_fmt(v) for v in r))
    return lines


def _fmt(v):
    v = float(v)
    if np.isinf(v):
        return "inf" if v > 0 else "-inf"
    if np.isnan(v):
        return "nan" if not np.signbit(v) else "-nan"
    return "%.9g" % v
