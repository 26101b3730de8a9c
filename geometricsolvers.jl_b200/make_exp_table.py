"""Writes csrc/gsb_exp_table.h: the 128 values 2^(j/128), j = 0..127, each as the nearest double
(hi) and the nearest double to the remainder (lo), and the reduction constants of csrc/gsb_exp.h,
computed with Python's decimal module at 60 significant digits.

python geometricsolvers.jl_b200/make_exp_table.py
"""

import math
import os
from decimal import Decimal, getcontext

getcontext().prec = 60
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "csrc", "gsb_exp_table.h")


def nearest(d: Decimal) -> float:
    """The double nearest to d (float() of a Decimal rounds correctly)."""
    return float(d)


def trim(v: float, bits: int) -> float:
    """v with its significand cut to `bits` bits (toward zero)."""
    m, e = math.frexp(v)
    scale = 2.0 ** bits
    return math.ldexp(math.floor(m * scale) / scale, e)


def main():
    ln2 = Decimal(2).ln()
    rows = []
    for j in range(128):
        t = (ln2 * j / 128).exp()
        hi = nearest(t)
        lo = nearest(t - Decimal(hi))
        rows.append((hi, lo))
    step = ln2 / 128
    # k * L1 is exact for |k| < 2^18 (|x| <= 746): L1 keeps 35 significant bits
    l1 = trim(nearest(step), 35)
    l2 = nearest(step - Decimal(l1))
    inv = nearest(Decimal(128) / ln2)
    with open(OUT, "w") as fh:
        fh.write("// Generated by make_exp_table.py: the table and constants of gsb_exp.h.\n")
        fh.write("#pragma once\n\n")
        fh.write(f"#define GSB_EXP_INV_STEP {inv.hex()}  /* 128 / ln 2 */\n")
        fh.write(f"#define GSB_EXP_STEP_HI {l1.hex()}  /* ln 2 / 128, 35 significant bits */\n")
        fh.write(f"#define GSB_EXP_STEP_LO {l2.hex()}  /* ln 2 / 128 - GSB_EXP_STEP_HI */\n\n")
        fh.write("/* 2^(j/128) = HI[j] + LO[j] */\n")
        for name, col in (("GSB_EXP_TABLE_HI", 0), ("GSB_EXP_TABLE_LO", 1)):
            fh.write(f"#define {name} {{ \\\n")
            for j in range(0, 128, 4):
                fh.write("    " + ", ".join(rows[q][col].hex() for q in range(j, j + 4)) + ", \\\n")
            fh.write("}\n")


if __name__ == "__main__":
    main()
