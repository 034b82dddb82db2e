"""Regenerates the golden fixtures in this folder from the reference's test data.

Run in a container where the reference is mounted at /root/reference:

    python tests/golden/make_golden.py

* convective_bc_gold.npy -- tests/data/convective_bc_gold.txt of the reference
  (the 1809 nodal temperatures of test_thermal_physics.hh:513-625, deal.II DoF
  order), stored as float64.
"""
import os
import sys

import numpy as np

REF = os.environ.get("ADAMANTINE_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    src = os.path.join(REF, "tests", "data", "convective_bc_gold.txt")
    if not os.path.exists(src):
        sys.exit(f"reference test data not found: {src}")
    vals = np.array([float(x) for x in open(src).read().split()], dtype=np.float64)
    assert vals.size == 1809, vals.size
    np.save(os.path.join(HERE, "convective_bc_gold.npy"), vals)
    print("wrote convective_bc_gold.npy", vals.size)


if __name__ == "__main__":
    main()
