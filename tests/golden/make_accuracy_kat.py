"""Extracts the reference's stored discretisation-error results into
accuracy_kat.json.

Source: staggered_grid/exec/stokes_preconditioner/test_gmres/run_result/
Accuracy_tests/{2d,3d}_dis_accuracy.dat of LowMachFHD -- the L0 norms of
f - A x_exact printed by main_driver.f90 (test_type = 0) for the Taylor
vortex (prob_sol = 1) and the prob_sol = 31 field, constant (prob_coeff = 1)
and smooth variable (prob_coeff = 5) coefficients, on 32, 64, 128 cells per
direction.  Only the "new code" section (apply_matrix) is taken; the later
"old code" section timed stag_applyop alone.

Run from the repository root with the reference checked out:
    python tests/golden/make_accuracy_kat.py /path/to/LowMachFHD
"""
import json
import os
import re
import sys

REL = "staggered_grid/exec/stokes_preconditioner/test_gmres/run_result/Accuracy_tests"


def parse(path, dim):
    rows = []
    coeff = sol = None
    viscs = None
    n = None
    cur = {}
    with open(path) as f:
        lines = f.readlines()
    for ln, line in enumerate(lines, 1):
        s = line.strip()
        if s.startswith("using old code"):
            break
        m = re.search(r"prob_coeff\s*=\s*(\d+)\s*,\s*prob_sol\s*=\s*(\d+)", s)
        if m:
            coeff, sol = int(m.group(1)), int(m.group(2))
            continue
        m = re.match(r"visc_type\s*=\s*(-?\d)(?:\s*or\s*(-?\d))?", s)
        if m:
            viscs = [int(m.group(1))] + ([int(m.group(2))] if m.group(2) else [])
            continue
        m = re.match(r"(\d+)\*\d+(?:\*\d+)?\s*mesh", s)
        if m:
            n = int(m.group(1))
            cur = {}
            continue
        m = re.search(r"L0 ([UVWP])\s*=\s*([-+0-9.Ee]+)", s)
        if m and n is not None and viscs is not None:
            cur[m.group(1)] = float(m.group(2).replace("E", "e"))
            keys = ["U", "V", "W", "P"][: dim] if dim == 3 else ["U", "V"]
            want = keys + (["P"] if sol == 31 else [])
            if dim == 3:
                want = ["U", "V", "W", "P"]
            if all(k in cur for k in want):
                for v in viscs:
                    rows.append({"dim": dim, "n": n, "prob_coeff": coeff, "prob_sol": sol,
                                 "visc_type": v, "errors": {k: cur[k] for k in want},
                                 "source": f"{REL}/{os.path.basename(path)}:{ln}"})
                cur = {}
    return rows


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    rows = parse(os.path.join(root, REL, "2d_dis_accuracy.dat"), 2)
    rows += parse(os.path.join(root, REL, "3d_dis_accuracy.dat"), 3)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "accuracy_kat.json")
    with open(out, "w") as f:
        json.dump(rows, f, indent=1)
    print(f"wrote {len(rows)} rows to {out}")


if __name__ == "__main__":
    main()
