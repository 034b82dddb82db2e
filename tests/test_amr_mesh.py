"""Refined-mesh logic on the host (through the C ABI, no GPU) against the
independent restatement in oracle/amr_oracle.py: the leaves after
refine_mesh's beam-driven rounds and after explicit refine / coarsen flags,
the non-hanging nodes and every hanging-node constraint, exactly; plus the
invariants the constraints must have (partition of unity, reproduction of
the polynomials of the element's degree) and the 2:1 balance across faces
and edges."""
import itertools

import numpy as np
import pytest

import amr_oracle
from amr_cases import amr_test_config

from adamantine_b200.amr import AmrMesh


def oracle_lattice(o, max_level):
    f = float(1 << (max_level + 1))
    return np.array([[round(v * f) for v in o.positions[k]] for k in o.dof_keys], np.int64)


def assert_same_mesh(m, o, max_level):
    lv = m.leaves()
    ol = np.array(o.forest.sorted_leaves(), np.int32).reshape(-1, 4)
    assert lv.shape == ol.shape and (lv == ol).all()
    assert m.n_dofs == o.n_dofs
    assert m.n_nodes == len(o.positions)
    assert (m.dof_lattice() == oracle_lattice(o, max_level)).all()
    xyz, ptr, dof, w = m.constraints()
    keys = sorted(o.hanging, key=lambda k: (k[2], k[1], k[0]))
    assert len(keys) == len(xyz)
    f = float(1 << (max_level + 1))
    for h, k in enumerate(keys):
        assert tuple(xyz[h]) == tuple(round(v * f) for v in o.positions[k])
        mine = dict(zip(dof[ptr[h]:ptr[h + 1]].tolist(), w[ptr[h]:ptr[h + 1]].tolist()))
        ref = {d: v for d, v in o.hanging[k].items() if abs(v) > 1e-14}
        assert set(mine) == set(ref)
        for d in mine:
            assert abs(mine[d] - ref[d]) <= 1e-15


@pytest.mark.parametrize("degree", [1, 2])
@pytest.mark.parametrize("n_ref", [1, 2])
def test_beam_refinement_matches_oracle(degree, n_ref):
    cfg = amr_test_config(degree=degree, n_cells=(4, 4, 2))
    m = AmrMesh(cfg, n_ref)
    o = amr_oracle.AmrProblem(cfg, n_ref)
    m.refine_mesh(0.0, 200e-6, 200, n_ref)
    o.refine_mesh_flags(0.0, 200e-6, 200, n_ref, False)
    o.build()
    assert m.leaves()[:, 0].max() == n_ref
    assert_same_mesh(m, o, n_ref)


@pytest.mark.parametrize("degree", [1, 2])
def test_refinement_then_coarsening_after_the_beam(degree):
    """coarsen_after_beam: the first window's cells coarsen once the beam has
    moved on (demo_316_short_amr.info refines every 5 steps this way)."""
    cfg = amr_test_config(degree=degree, n_cells=(6, 6, 2))
    m = AmrMesh(cfg, 2)
    o = amr_oracle.AmrProblem(cfg, 2)
    for t0 in (0.0, 60e-6, 120e-6, 180e-6):
        m.refine_mesh(t0, t0 + 30e-6, 30, 2, True)
        o.refine_mesh_flags(t0, t0 + 30e-6, 30, 2, True)
        o.build()
        assert_same_mesh(m, o, 2)
    # the region near the path's start went back to level 0
    lv = m.leaves()
    start = (lv[:, 0] == 0) & (lv[:, 1] == 2) & (lv[:, 2] == 2)
    assert start.any()


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_flags_match_oracle(seed):
    """Explicit refine / coarsen flags drawn at random, three rounds: the
    refinement, the balance-preserving coarsening and the balancing agree."""
    rng = np.random.default_rng(seed)
    cfg = amr_test_config(degree=2, n_cells=(3, 3, 2))
    L = 3
    m = AmrMesh(cfg, L)
    o = amr_oracle.AmrProblem(cfg, L)
    for _ in range(3):
        lv = [tuple(int(v) for v in c) for c in m.leaves()]
        ref = {c for c in lv if c[0] < L and rng.uniform() < 0.25}
        crs = {c for c in lv if c[0] > 0 and rng.uniform() < 0.6}
        m.execute(ref, crs)
        o.forest.execute(ref, crs)
        o.build()
        assert_same_mesh(m, o, L)


def test_inactive_coarse_cells_have_no_nodes_or_constraints():
    cfg = amr_test_config(degree=2, n_cells=(4, 4, 2))
    active = np.ones(32, np.uint8)
    active[16:] = 0  # the upper layer carries no material
    active[5] = 0
    m = AmrMesh(cfg, 2, active=active)
    o = amr_oracle.AmrProblem(cfg, 2, active=active)
    m.refine_mesh(0.0, 200e-6, 200, 2)
    o.refine_mesh_flags(0.0, 200e-6, 200, 2, False)
    o.build()
    assert_same_mesh(m, o, 2)
    # every DoF lies in the closure of the active region (z <= half height)
    lat = m.dof_lattice()
    assert lat[:, 2].max() <= 1 << 3


@pytest.mark.parametrize("degree", [1, 2])
def test_constraints_reproduce_polynomials(degree):
    """A hanging node's value, formed from its masters, equals the value of
    every polynomial of the element's degree in each variable at the node."""
    cfg = amr_test_config(degree=degree, n_cells=(4, 4, 2))
    m = AmrMesh(cfg, 2)
    m.refine_mesh(0.0, 200e-6, 200, 2)
    lat = m.dof_lattice().astype(float)
    xyz, ptr, dof, w = m.constraints()
    assert len(xyz) > 0
    h = xyz.astype(float)
    for e in itertools.product(range(degree + 1), repeat=3):
        f = lambda p: p[:, 0] ** e[0] * p[:, 1] ** e[1] * p[:, 2] ** e[2]
        fd, fh = f(lat / 8.0), f(h / 8.0)
        got = np.array([np.dot(w[ptr[i]:ptr[i + 1]], fd[dof[ptr[i]:ptr[i + 1]]]) for i in range(len(h))])
        assert np.allclose(got, fh, rtol=1e-13, atol=1e-13 * max(1.0, np.abs(fh).max()))
    sums = np.add.reduceat(w, ptr[:-1])
    assert np.allclose(sums, 1.0, atol=1e-14)


def test_balance_across_faces_and_edges():
    cfg = amr_test_config(degree=1, n_cells=(3, 3, 2))
    m = AmrMesh(cfg, 3)
    rng = np.random.default_rng(7)
    for _ in range(3):
        lv = [tuple(int(v) for v in c) for c in m.leaves()]
        m.execute({c for c in lv if c[0] < 3 and rng.uniform() < 0.3}, None)
    lv = m.leaves()
    L = 3
    # paint every leaf on the finest grid, then compare neighbours
    n = [c << L for c in (3, 3, 2)]
    level = np.zeros((n[2], n[1], n[0]), np.int32)
    for l, i, j, k in lv:
        s = 1 << (L - l)
        level[k * s:(k + 1) * s, j * s:(j + 1) * s, i * s:(i + 1) * s] = l
    assert level.max() == 3
    for o in amr_oracle.FACE_EDGE:
        a = level[max(0, o[2]):n[2] + min(0, o[2]), max(0, o[1]):n[1] + min(0, o[1]), max(0, o[0]):n[0] + min(0, o[0])]
        b = level[max(0, -o[2]):n[2] + min(0, -o[2]), max(0, -o[1]):n[1] + min(0, -o[1]),
                  max(0, -o[0]):n[0] + min(0, -o[0])]
        assert np.abs(a - b).max() <= 1


def test_bad_arguments_are_rejected():
    from adamantine_b200._lib import AdmError

    cfg = amr_test_config(degree=3)
    with pytest.raises(AdmError):
        AmrMesh(cfg, 1)  # degree 3 is not built on the GPU path
    cfg = amr_test_config(degree=2)
    with pytest.raises(AdmError):
        AmrMesh(cfg, 7)
    m = AmrMesh(cfg, 1)
    with pytest.raises(AdmError):
        m.refine_mesh(0.0, 1e-4, 10, 2)  # more rounds than levels
