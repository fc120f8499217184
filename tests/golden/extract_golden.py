"""Extract the reference's known-answer outputs into committed fixtures.

Reads, from the reference checkout, the expected outputs of its own tests:
  tests/tp_01.output        2-D slab solves: FGMRES totals and error norms
  tests/tp_02.output        time-weight and wave-condensation matrices
  tests/transfer_02.output  time prolongation / restriction / projection
and writes tests/golden/tp_01.json, tp_02.txt and transfer_02.txt.
Run once where the reference is mounted:
  python tests/golden/extract_golden.py /path/to/reference
"""
import json
import os
import re
import sys

# tests/tp_01.cc:781-806 runs these parameter files in this order; the
# settings are those of tests/json/tf01..tf08.json.
SECTIONS = [
    ("tf01", "heat", "DG", 2, 1),
    ("tf02", "heat", "CGP", 2, 2),
    ("tf03", "heat", "DG", 1, 1),
    ("tf04", "heat", "CGP", 1, 2),
    ("tf05", "wave", "DG", 4, 1),
    ("tf06", "wave", "CGP", 4, 2),
    ("tf07", "wave", "DG", 1, 1),
    ("tf08", "wave", "CGP", 1, 2),
]
N_DEG, N_REF, R0 = 3, 4, 2


def parse_tp01(text):
    its = [(int(a), int(b)) for a, b in
           re.findall(r"Average GMRES iterations \S+ \((\d+) gmres_iterations / (\d+) timesteps\)", text)]
    rows = re.findall(r"^\s*(\d+)\s+(\d+)\s+(\d+)\s+(\d+)\s+(\d+)\s+([0-9.e+-]+)\s+\S+\s+([0-9.e+-]+)\s+\S+\s+([0-9.e+-]+)",
                      text, re.M)
    assert len(its) == len(rows) == len(SECTIONS) * N_DEG * N_REF, (len(its), len(rows))
    out, i = [], 0
    for name, problem, ttype, steps, k0 in SECTIONS:
        for k in range(k0, k0 + N_DEG):
            for r in range(R0, R0 + N_REF):
                cells, sdofs, tdofs, stdofs, work, l8, l2, h1 = rows[i]
                out.append(dict(section=name, problem=problem, type=ttype, steps=steps, k=k, refine=r,
                                cells=int(cells), s_dofs=int(sdofs), t_dofs=int(tdofs),
                                iterations=its[i][0], slabs=its[i][1],
                                linf=float(l8), l2=float(l2), h1=float(h1)))
                i += 1
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/extract_golden.py /path/to/reference")
    ref = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(ref, "tests", "tp_01.output")) as f:
        rows = parse_tp01(f.read())
    with open(os.path.join(here, "tp_01.json"), "w") as f:
        json.dump(rows, f, indent=0)
    for name in ("tp_02", "transfer_02"):
        with open(os.path.join(ref, "tests", name + ".output")) as f:
            text = f.read()
        with open(os.path.join(here, name + ".txt"), "w") as f:
            f.write(text)
    print("wrote", len(rows), "tp_01 rows")


if __name__ == "__main__":
    main()
