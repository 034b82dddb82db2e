"""Regenerates the golden fixtures in this folder from the reference's test data.

Give the reference's source tree as the argument (or in the environment
variable ADAMANTINE_REFERENCE):

    python tests/golden/make_golden.py <adamantine source tree>

* convective_bc_gold.npy -- tests/data/convective_bc_gold.txt of the reference
  (the 1809 nodal temperatures of test_thermal_physics.hh:513-625, deal.II DoF
  order), stored as float64.
* deposition_inputs.npz -- the inputs of test_material_deposition.cc:
  scan_path.txt and scan_path_L.txt as (end_time, power_modifier, x, y, z)
  segment rows (ScanPath "segment" format: mode 1 = point held for `param`
  seconds, mode 0 = line at `param` m/s), and the box file
  material_path_test_material_deposition.txt as rows (center[3], size[3],
  time, angle).
* microstructure_G_R_gold_1.txt, microstructure_G_R_gold_2.txt -- the gold
  files of test_microstructure.cc (one 10 mm x 10 mm Q2 cell, liquidus 100,
  old field 1000 (+ (x - 1)^2 + y^2 in the second), new field 50 (+ the
  same), delta_t 1.1), copied line by line.
* integration_3d_gold.txt -- tests/data/integration_3d_gold.txt of the
  reference: the 26177 temperatures (4 significant digits, deal.II DoF
  order) after 100 forward Euler steps of demo_316_short_anisotropic.info
  (test_integration_3d.cc:112-115), copied as is; and
  integration_3d_scan_path.npy, the segments of demo_316_short_scan_path.txt
  as (end_time, power_modifier, x, y, z) rows.
* amr_test_scan_path.npy -- the segments of bare_plate_L_scan_path_fast.txt,
  the scan path of amr_test.info (test_integration_3d_amr.cc:19-58: 4 x 4 x 1
  FE_Q(3) cells of 5 x 5 x 0.5 mm, one refinement along the beam every 200
  steps, 250 forward Euler steps of 1 us; expected max 329.5 K, min 296.1 K),
  as (end_time, power_modifier, x, y, z) rows.
* demo_316_short_amr_scan_path.npy -- the segments of
  demo_316_short_scan_path_amr.txt, the scan path of demo_316_short_amr.info
  (test_integration_3d_amr.cc:60-88: 25 x 25 x 2 FE_Q(2) cells of 5 x 5 x
  0.5 mm, refinement every 5 steps with coarsening after the beam, 40
  forward Euler steps of 1e-4 s; expected 13005 DoFs at the end), as
  (end_time, power_modifier, x, y, z) rows.
* integration_3d_gold_short.npz -- tests/data/integration_3d_gold_short.txt
  (229570 temperatures, 6 significant digits, stored as float32, exact to
  the printed digits) of demo_316_short.info (test_integration_3d.cc:117-120:
  50 x 50 x 8 FE_Q(3), convective and radiative faces, 67 forward Euler
  steps of 6e-5 s).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = None


def main():
    global REF
    REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ADAMANTINE_REFERENCE")
    if not REF:
        sys.exit("usage: make_golden.py <adamantine source tree> (or set ADAMANTINE_REFERENCE)")
    src = os.path.join(REF, "tests", "data", "convective_bc_gold.txt")
    if not os.path.exists(src):
        sys.exit(f"reference test data not found: {src}")
    vals = np.array([float(x) for x in open(src).read().split()], dtype=np.float64)
    assert vals.size == 1809, vals.size
    np.save(os.path.join(HERE, "convective_bc_gold.npy"), vals)
    print("wrote convective_bc_gold.npy", vals.size)

    data = os.path.join(REF, "tests", "data")
    out = {}
    for name in ("scan_path", "scan_path_L"):
        out[name] = segments(open(os.path.join(data, name + ".txt")).read())
    lines = open(os.path.join(data, "material_path_test_material_deposition.txt")).read().split("\n")
    assert int(lines[0]) == 3
    out["material_path"] = np.array([[float(v) for v in ln.split()] for ln in lines[1:] if ln.strip()])
    np.savez(os.path.join(HERE, "deposition_inputs.npz"), **out)
    print("wrote deposition_inputs.npz", {k: v.shape for k, v in out.items()})

    src = os.path.join(data, "integration_3d_gold.txt")
    vals = open(src).read().split()
    assert len(vals) == 26177, len(vals)
    with open(os.path.join(HERE, "integration_3d_gold.txt"), "w") as fh:
        fh.write(" ".join(vals) + "\n")
    np.save(os.path.join(HERE, "integration_3d_scan_path.npy"),
            np.array(segments(open(os.path.join(data, "demo_316_short_scan_path.txt")).read())))
    print("wrote integration_3d_gold.txt", len(vals), "and integration_3d_scan_path.npy")
    short = np.array([float(v) for v in open(os.path.join(data, "integration_3d_gold_short.txt")).read().split()])
    assert short.size == 229570, short.size
    np.savez_compressed(os.path.join(HERE, "integration_3d_gold_short.npz"), values=short.astype(np.float32))
    print("wrote integration_3d_gold_short.npz", short.size)

    np.save(os.path.join(HERE, "amr_test_scan_path.npy"),
            segments(open(os.path.join(data, "bare_plate_L_scan_path_fast.txt")).read()))
    print("wrote amr_test_scan_path.npy")
    np.save(os.path.join(HERE, "demo_316_short_amr_scan_path.npy"),
            segments(open(os.path.join(data, "demo_316_short_scan_path_amr.txt")).read()))
    print("wrote demo_316_short_amr_scan_path.npy")

    for k in (1, 2):
        name = f"microstructure_G_R_gold_{k}.txt"
        lines = [ln for ln in open(os.path.join(data, name)).read().split("\n") if ln.strip()]
        with open(os.path.join(HERE, name), "w") as fh:
            fh.write("\n".join(lines) + "\n")
        print("wrote", name, len(lines))


def segments(text):
    """ScanPath segment-format text -> (end_time, power_modifier, x, y, z) rows
    (the first row is the start point)."""
    rows = [ln.split() for ln in text.split("\n")[3:] if ln.strip()]
    out = []
    t = 0.0
    prev = None
    for r in rows:
        mode, x, y, z, pmod, param = int(r[0]), float(r[1]), float(r[2]), float(r[3]), float(r[4]), float(r[5])
        if mode == 1 or prev is None:
            t = t + param
        else:
            t = t + float(np.sqrt((x - prev[0]) ** 2 + (y - prev[1]) ** 2 + (z - prev[2]) ** 2)) / param
        out.append([t, pmod, x, y, z])
        prev = (x, y, z)
    return np.array(out)


if __name__ == "__main__":
    main()
