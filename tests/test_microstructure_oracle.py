"""CPU pins of the microstructure restatement against the reference's own gold
files (tests/test_microstructure.cc: one 10 mm x 10 mm FE_Q(2) cell, liquidus
100, delta_t 1.1)."""
import os

import numpy as np

from microstructure_oracle import compute_G_and_R, format_records, nodal_derivative

HERE = os.path.dirname(os.path.abspath(__file__))


def gold(k):
    return [ln for ln in open(os.path.join(HERE, "golden", f"microstructure_G_R_gold_{k}.txt")).read().split("\n")
            if ln.strip()]


def unit_cell_fields(extra):
    x = np.linspace(0.0, 10e-3, 3)
    X, Y = np.meshgrid(x, x)  # [y][x]
    f = (X - 1.0) ** 2 + Y ** 2 if extra else np.zeros_like(X)
    return 1000.0 + f, 50.0 + f


def test_uniform_fields_match_gold_1():
    """G = 0 everywhere, so R is inf; the cooling rate is 1000 - 50 / 1.1."""
    t_old, t_new = unit_cell_fields(False)
    rec = compute_G_and_R((1, 1), (10e-3, 10e-3), 2, t_old, t_new, 1.1, [100.0])
    assert format_records(rec) == gold(1)


def test_quadratic_fields_match_gold_2():
    t_old, t_new = unit_cell_fields(True)
    rec = compute_G_and_R((1, 1), (10e-3, 10e-3), 2, t_old, t_new, 1.1, [100.0])
    assert format_records(rec) == gold(2)


def test_cooling_rate_keeps_the_reference_precedence():
    """old - new / dt, not (old - new) / dt."""
    t_old, t_new = unit_cell_fields(False)
    rec = compute_G_and_R((1, 1), (10e-3, 10e-3), 2, t_old, t_new, 1.1, [100.0])
    assert np.allclose(rec[:, 3], 1000.0 - 50.0 / 1.1, rtol=0, atol=1e-12)


def test_nodal_derivative_is_exact_on_quadratics():
    D = nodal_derivative(2)
    assert np.array_equal(D, [[-3.0, 4.0, -1.0], [-1.0, 0.0, 1.0], [1.0, -4.0, 3.0]])
    assert np.array_equal(nodal_derivative(1), [[-1.0, 1.0], [-1.0, 1.0]])


def test_3d_shared_nodes_give_one_record_per_cell_and_skip_inactive_cells():
    """Two cells along x; the whole field crosses the liquidus; the shared
    face's nodes appear once per cell (each cell's one-sided gradient);
    an inactive cell and a cell whose material has a higher liquidus write
    nothing."""
    n_cells, extent = (2, 1, 1), (2e-3, 1e-3, 1e-3)
    nodes = (5, 3, 3)
    z, y, x = np.meshgrid(*[np.linspace(0, e, n) for e, n in zip(extent[::-1], nodes[::-1])], indexing="ij")
    t_new = 50.0 + 1e4 * x ** 2 + 3e3 * y - 2e3 * z
    t_old = t_new + 900.0
    rec = compute_G_and_R(n_cells, extent, 2, t_old, t_new, 0.5, [100.0, 2000.0])
    assert rec.shape == (54, 6)
    shared = rec[np.isclose(rec[:, 0], 1e-3)]
    assert len(shared) == 18
    # the x-derivative of a quadratic is exact on each side
    assert np.allclose(np.sqrt(shared[:, 3] ** 2 - (3e3 ** 2 + 2e3 ** 2)), 2e4 * 1e-3, rtol=1e-9)
    assert compute_G_and_R(n_cells, extent, 2, t_old, t_new, 0.5, [100.0], active=[1, 0]).shape == (27, 6)
    assert compute_G_and_R(n_cells, extent, 2, t_old, t_new, 0.5, [100.0, 2000.0], material=[0, 1]).shape == (27, 6)
