"""The CPU oracle with the driver's deposition window against the reference's
driver-level gold file (test_integration_3d.cc:112-115): the 26177
temperatures after 100 forward Euler steps of the anisotropic 3-D demo,
compared digit for digit in the file's own 4-significant-digit format, in
deal.II's DoF order on the final (partly activated) mesh."""
from dealii_order import dof_to_node
import numpy as np

from integration_demo import (BOX, SHORT_DT, SHORT_DURATION, demo_config, demo_short_config, gold_short, gold_text,
                              run_oracle)

from adamantine_b200.deposition import deposition_boxes


def test_oracle_reproduces_integration_3d_gold():
    cfg = demo_config()
    boxes = deposition_boxes(cfg, *BOX)
    y, active, n, _ = run_oracle(cfg, boxes)
    assert n == 100
    order = dof_to_node(3, cfg.geometry.n_cells, 2, active=active)
    gold = gold_text()
    assert len(order) == len(gold) == 26177  # the deposited cells' DoFs included
    mine = ["%.3e" % v for v in y[order]]
    assert mine == gold


def test_oracle_reproduces_integration_3d_short_gold():
    """demo_316_short.info (test_integration_3d.cc:117-120, which checks each
    value to a relative tolerance of 0.1): FE_Q(3), convective and radiative
    faces, deposition, 66 steps of 6e-5 s and a last one cut to 4e-5 s so
    that the run ends at the 4 ms duration (application/adamantine.hh
    :1110-1111); 229570 values. The DoF count is exact, 99.9 % of the values
    agree in all 6 printed digits and none differs by more than the printed
    precision (5e-6 relative)."""
    cfg = demo_short_config()
    boxes = deposition_boxes(cfg, *BOX)
    y, active, n, o = run_oracle(cfg, boxes, SHORT_DT, SHORT_DURATION)
    assert n == 67
    order = dof_to_node(3, cfg.geometry.n_cells, 3, active=active)
    gold = gold_short()
    assert len(order) == len(gold) == 229570
    v = y[order]
    rel = np.abs(v - gold) / np.abs(gold)
    assert rel.max() <= 0.1  # the reference test's own tolerance
    assert rel.max() <= 5e-6
    assert np.mean(["%g" % a == "%g" % b for a, b in zip(v, gold)]) >= 0.999
