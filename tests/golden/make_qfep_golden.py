"""Golden outputs of the reference's own Python free-energy estimators
(src/Qgpu/calc.py: EXPfwd, EXPbwd, overlap_sampling, BAR) for the qfep
restatement's tests.

calc.py imports a sibling module at its top, so this script takes the four
functions' own source out of the file (ast) and runs them unchanged on seeded
energy series; it stores inputs and outputs in qgpu_calc_estimators.json.
Run here, where the reference tree exists:

    python tests/golden/make_qfep_golden.py /path/to/reference
"""
import ast
import json
import math
import os
import sys

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "qgpu_calc_estimators.json")
NAMES = ("EXPfwd", "EXPbwd", "overlap_sampling", "BAR")


def functions(path):
    text = open(path).read()
    tree = ast.parse(text)
    ns = {"math": math, "np": np}
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name in NAMES:
            exec(ast.get_source_segment(text, node), ns)
    return ns


def main(ref: str):
    ns = functions(os.path.join(ref, "src", "Qgpu", "calc.py"))
    rng = np.random.default_rng(2024)
    cases = []
    for k in range(6):
        n = int(rng.integers(20, 80))
        kT = float(rng.uniform(0.55, 0.65))
        l1 = [float(x) for x in (1.0 - 0.1 * k, 0.1 * k)]
        l2 = [float(x) for x in (0.9 - 0.1 * k, 0.1 + 0.1 * k)]
        constant = k < 4
        if constant:
            # every record of the window the same: the case where the calc.py
            # estimators and qfep's are related exactly
            row = rng.normal(0.0, 3.0, 2)
            series = np.tile(row, (n, 1))
        else:
            series = rng.normal(0.0, 3.0, (n, 2)) + np.array([0.0, 1.5])
        MA1 = series.tolist()
        fwd = ns["EXPfwd"](MA1, l1, l2, kT, 0)
        bwd = ns["EXPbwd"](MA1, l1, l2, kT, 0)
        os_ = ns["overlap_sampling"](MA1, l1, l2, kT, 0)
        bar = ns["BAR"](MA1, l1, l2, kT, 0, os_ if os_ != 0 else 0.1)
        cases.append({"constant": constant, "kT": kT, "l1": l1, "l2": l2, "series": MA1,
                      "EXPfwd": fwd, "EXPbwd": bwd, "overlap_sampling": os_, "BAR": bar})
    json.dump({"source": "src/Qgpu/calc.py EXPfwd, EXPbwd, overlap_sampling, BAR (run unchanged)",
               "cases": cases}, open(OUT, "w"), indent=0)
    print("wrote", OUT)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_qfep_golden.py /path/to/reference")
    main(sys.argv[1])
