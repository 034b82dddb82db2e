"""The refined-mesh restatement (oracle/amr_oracle.py) pinned to the
reference and checked for the structure the constrained operator must have.

* The reference's amr_test.info (test_integration_3d_amr.cc:19-58), FE_Q(3),
  one level of refinement along the beam before step 1 and at step 200, 250
  forward Euler steps: the reference expects max 329.5 K and min 296.1 K
  with a 10 % tolerance; the restatement lands within 0.1 % of both.
* Refining every cell gives the uniform level-1 grid: the constrained
  operator then equals the uniform oracle's.
* With temperature-independent properties (linear conduction) the
  constrained operator C^T A C is symmetric, which holds only if the
  prolongation and the restriction are transposes of each other.
"""
import numpy as np
import pytest

import amr_oracle
from amr_cases import AMR_MAX, AMR_MIN, amr_test_config, run_amr
from oracle_py import Oracle


def test_reference_amr_test_extremes():
    cfg = amr_test_config(degree=3)
    o = amr_oracle.AmrProblem(cfg, 1, initial_state=cfg.geometry.initial_state())
    o.setup(300.0)
    run_amr(o)
    assert o.forest.L == 1 and max(c[0] for c in o.forest.leaves) == 1
    hi, lo = o.y.max(), o.y.min()
    # the reference's own tolerance, then the agreement actually reached
    assert abs(hi - AMR_MAX) <= 0.1 * AMR_MAX and abs(lo - AMR_MIN) <= 0.1 * AMR_MIN
    assert abs(hi - AMR_MAX) <= 1e-3 * AMR_MAX and abs(lo - AMR_MIN) <= 1e-3 * AMR_MIN


@pytest.mark.parametrize("degree", [1, 2])
def test_uniform_refinement_equals_the_fine_grid(degree):
    cfg = amr_test_config(degree=degree, n_cells=(3, 2, 2))
    o = amr_oracle.AmrProblem(cfg, 1)
    o.setup(300.0)
    o.execute(set(o.forest.leaves), set())
    assert all(c[0] == 1 for c in o.forest.leaves) and not o.hanging
    fine = amr_oracle.AmrProblem(amr_test_config(degree=degree, n_cells=(6, 4, 4)), 0)
    fine.setup(300.0)
    rng = np.random.default_rng(3)
    pts = o.dof_points()
    y = 400.0 + 1500.0 * np.exp(-((pts[:, 0] - 1.5) ** 2 + (pts[:, 1] - 1.0) ** 2) / 0.5) + rng.uniform(0, 5, len(pts))
    # the same field on the fine grid's DoFs (same positions, scaled by 2)
    fpts = fine.dof_points() / 2.0
    order = np.lexsort((fpts[:, 0], fpts[:, 1], fpts[:, 2]))
    mine = np.lexsort((pts[:, 0], pts[:, 1], pts[:, 2]))
    yf = np.empty_like(y)
    yf[order] = y[mine]
    for t in (0.0, 60e-6):
        o.set_time(t)
        fine.set_time(t)
        a = o.vmult(y)
        b = fine.vmult(yf)
        assert np.abs(a[mine] - b[order]).max() <= 1e-12 * np.abs(b).max()
    assert np.allclose(o.inv_mass[mine], fine.inv_mass[order], rtol=1e-14, atol=0)


@pytest.mark.parametrize("degree", [1, 2])
def test_constrained_operator_is_symmetric_for_linear_conduction(degree):
    cfg = amr_test_config(degree=degree, n_cells=(4, 4, 2), n_states=1)
    o = amr_oracle.AmrProblem(cfg, 2)
    o.setup(300.0)
    o.refine_mesh(0.0, 200e-6, 200, 2)
    assert o.hanging
    o.set_time(1.0)  # after the scan path: no source
    rng = np.random.default_rng(11)
    x = 300.0 + rng.uniform(0, 500, o.n_dofs)
    z = 300.0 + rng.uniform(0, 500, o.n_dofs)
    ax, az = o.vmult(x), o.vmult(z)
    assert abs(z @ ax - x @ az) <= 1e-12 * abs(z @ ax)
    # the constant field is in the kernel of the conduction operator
    assert np.abs(o.vmult(np.full(o.n_dofs, 700.0))).max() <= 1e-9 * np.abs(ax).max()


def test_reference_demo_316_short_amr_dof_count():
    """demo_316_short_amr.info (test_integration_3d_amr.cc:60-88): FE_Q(2),
    refinement along the beam every 5 steps with coarsening after it, 40
    forward Euler steps of 1e-4 s. The reference expects 13005 DoFs at the
    end (the beam is off after 2.8 ms and the mesh has coarsened back to the
    25 x 25 x 2 grid's 51 x 51 x 5 nodes) and a finite field; the refined
    meshes on the way have more."""
    from amr_cases import (DEMO_AMR_DOFS, DEMO_AMR_DT, DEMO_AMR_DURATION, DEMO_AMR_EVERY,
                           demo_316_short_amr_config)

    cfg = demo_316_short_amr_config()
    o = amr_oracle.AmrProblem(cfg, 1, initial_state=cfg.geometry.initial_state())
    o.setup(300.0)
    seen = []
    run_amr(o, dt=DEMO_AMR_DT, duration=DEMO_AMR_DURATION, every=DEMO_AMR_EVERY, n_refinements=1, coarsen=True,
            on_step=lambda n, t: seen.append(o.n_dofs))
    assert o.n_dofs == DEMO_AMR_DOFS
    assert np.isfinite(o.y).all()
    assert max(seen) > DEMO_AMR_DOFS  # it was refined on the way
