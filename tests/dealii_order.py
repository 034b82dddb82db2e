"""deal.II DoF enumeration on an unrefined box -- test infrastructure.

The reference's gold files are stored in deal.II's DoF order.  For a
subdivided_hyper_rectangle without refinement, DoFHandler::distribute_dofs
walks the cells in creation (lexicographic) order and, on each cell, numbers
the not-yet-numbered DoFs of its vertices, then its lines, then its quads, then
its interior, using deal.II's GeometryInfo numbering of those objects.  This
module restates that walk for FE_Q(1), FE_Q(2) and (3-D) FE_Q(3) and
returns, for every
deal.II DoF, the node index of the full-grid lexicographic numbering.
"""
import itertools

import numpy as np

# GeometryInfo<3>: lines as (vertex a, vertex b); vertex v = ix + 2*iy + 4*iz
_LINES_3D = [(0, 2), (1, 3), (0, 1), (2, 3), (4, 6), (5, 7), (4, 5), (6, 7), (0, 4), (1, 5), (2, 6), (3, 7)]
_LINES_2D = [(0, 2), (1, 3), (0, 1), (2, 3)]  # the faces of a quad


def _vcoord(v, dim):
    return [(v >> d) & 1 for d in range(dim)]


def dof_to_node(dim, n_cells, degree, active=None):
    """active: per cell (lexicographic), or None for all. Cells without
    degrees of freedom (FE_Nothing, inactive) are skipped by the walk, so the
    DoFs of an hp mesh are those of its active cells in the same order."""
    nc = list(n_cells[:dim])
    nn = [degree * n + 1 for n in nc]

    def node(cc, loc):
        idx, mul = 0, 1
        for d in range(dim):
            idx += (degree * cc[d] + loc[d]) * mul
            mul *= nn[d]
        return idx

    objects = []  # local node offsets (0..degree per axis) of each DoF, in order
    for v in range(2 ** dim):
        objects.append([degree * c for c in _vcoord(v, dim)])
    if degree == 3 and dim == 3:
        # two DoFs per line, from its first vertex to its second; four per
        # face, lexicographic in the face's own coordinates (faces 0/1:
        # (y, z), 2/3: (z, x), 4/5: (x, y)); eight inside, lexicographic
        for a, b in _LINES_3D:
            ca, cb = _vcoord(a, dim), _vcoord(b, dim)
            d = [k for k in range(3) if ca[k] != cb[k]][0]
            for j in (1, 2):
                loc = [3 * c for c in ca]
                loc[d] = j
                objects.append(loc)
        face_axes = {0: (1, 2), 1: (2, 0), 2: (0, 1)}
        for f in range(6):
            d, side = divmod(f, 2)
            u, w = face_axes[d]
            for jw in (1, 2):
                for ju in (1, 2):
                    loc = [0, 0, 0]
                    loc[d] = 3 * side
                    loc[u] = ju
                    loc[w] = jw
                    objects.append(loc)
        for k in (1, 2):
            for j in (1, 2):
                for i in (1, 2):
                    objects.append([i, j, k])
    if degree == 2:
        lines = _LINES_3D if dim == 3 else _LINES_2D
        for a, b in lines:
            ca, cb = _vcoord(a, dim), _vcoord(b, dim)
            objects.append([ca[d] + cb[d] for d in range(dim)])
        if dim == 3:
            for f in range(6):
                d, side = divmod(f, 2)
                loc = [1, 1, 1]
                loc[d] = 2 * side
                objects.append(loc)
        objects.append([1] * dim)
    order, seen = [], set()
    for ci, cell_rev in enumerate(itertools.product(*[range(n) for n in reversed(nc)])):
        if active is not None and not active[ci]:
            continue
        cc = list(reversed(cell_rev))
        for loc in objects:
            g = node(cc, loc)
            if g not in seen:
                seen.add(g)
                order.append(g)
    return np.array(order, dtype=np.int64)
