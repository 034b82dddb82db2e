"""The CPU oracle with the driver's deposition window against the reference's
driver-level gold file (test_integration_3d.cc:112-115): the 26177
temperatures after 100 forward Euler steps of the anisotropic 3-D demo,
compared digit for digit in the file's own 4-significant-digit format, in
deal.II's DoF order on the final (partly activated) mesh."""
from dealii_order import dof_to_node
from integration_demo import BOX, demo_config, gold_text, run_oracle

from adamantine_b200.deposition import deposition_boxes


def test_oracle_reproduces_integration_3d_gold():
    cfg = demo_config()
    boxes = deposition_boxes(cfg, *BOX)
    y, active, n = run_oracle(cfg, boxes)
    assert n == 100
    order = dof_to_node(3, cfg.geometry.n_cells, 2, active=active)
    gold = gold_text()
    assert len(order) == len(gold) == 26177  # the deposited cells' DoFs included
    mine = ["%.3e" % v for v in y[order]]
    assert mine == gold
