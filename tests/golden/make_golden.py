"""Generates tests/golden/standard_newton_lu_f64.json from the reference's golden table.

python tests/golden/make_golden.py <path of GeometricSolvers.jl's
    test/verification/standard_reference.csv>

It keeps the Float64 rows of the columns in COLUMNS (code, iterations, f_evals, fnorm and the
unstable/platform flags) and adds each cell's start, restated from
test/helpers/standard_problems.jl:386-424 (u0, and 10 u0 and 100 u0 where they differ from an
earlier start, test/helpers/standard_problems.jl:44-52).
"""

import csv
import json
import os
import sys
from fractions import Fraction

COLUMNS = ("Newton Static LU", "Newton Backtracking LU", "Newton Backtracking QR",
           "Newton DogLeg LU", "Newton reuse 3 Backtracking LU")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "standard_newton_lu_f64.json")


def u0(number):
    """The start of each problem in Float64 (test/helpers/standard_problems.jl:386-424)."""
    f = float
    return {
        1: [-1.2] + [1.0] * 9,
        2: [3.0, -1.0, 0.0, 1.0],
        3: [0.0, 1.0],
        4: [-3.0, -1.0, -3.0, -1.0],
        5: [-1.0, 0.0, 0.0],
        6: [0.0, 0.0],
        7: [f(Fraction(2 * i - 2, 3)) for i in (1, 2)],
        8: [0.5] * 10,
        9: [f(Fraction(i * (i - 11), 121)) for i in range(1, 11)],
        10: [f(Fraction(i * (i - 11), 121)) for i in range(1, 11)],
        11: [0.1] * 10,
        12: [1.0 - i / 10 for i in range(1, 11)],
        13: [-1.0] * 10,
        14: [-1.0] * 10,
        15: [1.0, 0.0, 0.0, 1.0],
        16: [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0],
        17: [1.0, 5.0],
        18: [2.0, 2.0],
        19: [3.0, 3.0],
        20: [1.0],
        21: [0.5, -2.0],
        22: [1.0, 0.0],
        23: [1.0] * 10,
    }[number]


def starts(number):
    x = u0(number)
    out = [("u0", x)]
    for label, s in (("10u0", 10), ("100u0", 100)):
        y = [s * v for v in x]
        if not any(y == z for _, z in out):
            out.append((label, y))
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    rows = {}
    with open(sys.argv[1]) as fh:
        for r in csv.DictReader(fh):
            if r["eltype"] != "Float64":
                continue
            if r["column"] not in COLUMNS:
                continue
            rows[(int(r["problem"]), r["start"], r["column"])] = r
    cells = []
    for number in range(1, 24):
        for label, x0 in starts(number):
            for column in COLUMNS:
                r = rows[(number, label, column)]
                cells.append({
                    "problem": number, "start": label, "x0": x0, "column": column,
                    "code": r["code"], "iterations": int(r["iterations"]),
                    "f_evals": int(r["f_evals"]), "fnorm": float(r["fnorm"]),
                    "unstable": r["unstable"] == "true", "platform": r["platform"] == "true",
                })
    assert len(cells) == 67 * len(COLUMNS), len(cells)
    with open(OUT, "w") as fh:
        json.dump({"source": "test/verification/standard_reference.csv", "cells": cells}, fh, indent=1)
    print(f"wrote {len(cells)} cells to {OUT}")


if __name__ == "__main__":
    main()
