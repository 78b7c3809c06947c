"""Writes dft_consts.h: cos/sin of 2*pi*m/R for every codelet radix R.

Run from this directory: `python gen_consts.py`.  The values are the double
nearest to each constant (a 60-digit Taylor series rounded once).  The constants are returned by a
switch so that a fully unrolled codelet folds them into immediates.
"""
import os
from decimal import Decimal, getcontext

getcontext().prec = 60
_PI = Decimal("3.14159265358979323846264338327950288419716939937510582097494459")


def _cos_sin(m: int, r: int):
    """cos/sin(2*pi*m/r) to 60 digits (Taylor series), rounded once to double."""
    x = 2 * _PI * Decimal(m) / Decimal(r)
    # reduce to [-pi, pi]
    while x > _PI:
        x -= 2 * _PI
    c, s = Decimal(0), Decimal(0)
    term = Decimal(1)
    k = 0
    while True:
        if k % 4 == 0:
            c += term
        elif k % 4 == 1:
            s += term
        elif k % 4 == 2:
            c -= term
        else:
            s -= term
        k += 1
        term = term * x / k
        if abs(term) < Decimal("1e-55"):
            break
    c = Decimal(0) if abs(c) < Decimal("1e-40") else c
    s = Decimal(0) if abs(s) < Decimal("1e-40") else s
    return float(c), float(s)

RADICES = list(range(2, 17)) + [32]


def main() -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    out = [
        "// Generated by gen_consts.py: cos/sin(2*pi*m/R), m < R, for each codelet radix.",
        "#pragma once",
        "",
        "__host__ __device__ __forceinline__ constexpr double dft_cos(int r, int m) {",
        "  switch (r * 64 + m) {",
    ]
    for r in RADICES:
        for m in range(r):
            out.append(f"    case {r * 64 + m}: return {_cos_sin(m, r)[0]!r};")
    out += ["    default: return 0.0;", "  }", "}", ""]
    out += [
        "__host__ __device__ __forceinline__ constexpr double dft_sin(int r, int m) {",
        "  switch (r * 64 + m) {",
    ]
    for r in RADICES:
        for m in range(r):
            out.append(f"    case {r * 64 + m}: return {_cos_sin(m, r)[1]!r};")
    out += ["    default: return 0.0;", "  }", "}", ""]
    with open(os.path.join(here, "dft_consts.h"), "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
