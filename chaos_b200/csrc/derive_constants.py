"""Derive the floating-point constants of the engine and of the oracle from their mathematical definitions.

Everything is computed in 100-digit decimal arithmetic and rounded once into binary64:

* pi/2 split into three doubles P1 + P2 + P3 (each the correctly rounded remainder of the one before), and
  2/pi, for the Cody-Waite argument reduction of sin / cos (Cody and Waite, "Software Manual for the Elementary
  Functions", 1980);
* the Taylor coefficients of sin and cos about 0 and of the atanh series of the logarithm, each correctly
  rounded;
* ln 2 split into a 42-bit head (so that e * LN2_HI is exact for every binary64 exponent e) and its rounded tail,
  for the logarithm;
* 1 / ln 2 and the Taylor coefficients 1 / n! of exp; atan(k / 16) for k = 0..16 split head + tail, the Taylor
  coefficients of atan, pi split head + tail, for this project's exp and atan2;
* the 3-stage Gauss-Legendre coefficients A and b in closed form (nodes 1/2 -+ sqrt(15)/10, 1/2), each split into
  a correctly rounded head and the rounded remainder, as src/Integrators/gauss.jl:21-26 (`_split`) does with its
  320-bit values; the collocation conditions sum_j A_ij c_j^(k-1) = c_i^k / k are checked to 1e-90.

pi comes from Machin's formula, ln 2 from the decimal module. Run it to (re)write
`chaos_b200/csrc/cl_constants.h` and `oracle/oracle_constants.hpp`; `tests/test_constants.py` re-derives the
values and checks both files.
"""
from __future__ import annotations

import math
import os
import sys
from decimal import Decimal, getcontext

getcontext().prec = 100


def _arctan_inv(n: int) -> Decimal:
    x = Decimal(1) / n
    x2 = x * x
    s = t = x
    k = 1
    while True:
        t = -t * x2
        k += 2
        d = t / k
        if abs(d) < Decimal(10) ** -98:
            return s
        s += d


def _arctan_frac(k: int, m: int) -> Decimal:
    """atan(k / m) for 0 <= k <= m by the series of atan(x) = sum (-1)^i x^(2i+1) / (2i+1) after two halvings of the
    angle, atan(x) = 2 atan(x / (1 + sqrt(1 + x^2)))."""
    if k == 0:
        return Decimal(0)
    x = Decimal(k) / m
    for _ in range(2):
        x = x / (1 + (1 + x * x).sqrt())
    x2 = x * x
    s = t = x
    i = 1
    while True:
        t = -t * x2
        i += 2
        d = t / i
        if abs(d) < Decimal(10) ** -98:
            return 4 * s
        s += d


def derive() -> dict[str, float]:
    pi = 16 * _arctan_inv(5) - 4 * _arctan_inv(239)
    pio2 = pi / 2
    c: dict[str, float] = {}
    c["CL_PIO2_1"] = float(pio2)
    r = pio2 - Decimal(c["CL_PIO2_1"])
    c["CL_PIO2_2"] = float(r)
    r -= Decimal(c["CL_PIO2_2"])
    c["CL_PIO2_3"] = float(r)
    c["CL_TWO_OVER_PI"] = float(2 / pi)
    ln2 = Decimal(2).ln()
    hi = Decimal(math.floor(ln2 * Decimal(2) ** 42)) / Decimal(2) ** 42
    c["CL_LN2_HI"] = float(hi)
    assert Decimal(c["CL_LN2_HI"]) == hi
    c["CL_LN2_LO"] = float(ln2 - hi)
    s15 = Decimal(15).sqrt()
    A = [[Decimal(5) / 36, Decimal(2) / 9 - s15 / 15, Decimal(5) / 36 - s15 / 30],
         [Decimal(5) / 36 + s15 / 24, Decimal(2) / 9, Decimal(5) / 36 - s15 / 24],
         [Decimal(5) / 36 + s15 / 30, Decimal(2) / 9 + s15 / 15, Decimal(5) / 36]]
    b = [Decimal(5) / 18, Decimal(4) / 9, Decimal(5) / 18]
    nodes = [Decimal(1) / 2 - s15 / 10, Decimal(1) / 2, Decimal(1) / 2 + s15 / 10]
    for i in range(3):
        for k in range(1, 4):
            lhs = sum(A[i][j] * nodes[j] ** (k - 1) for j in range(3))
            assert abs(lhs - nodes[i] ** k / k) < Decimal(10) ** -90
    for i in range(3):
        for j in range(3):
            h = float(A[i][j])
            c[f"CL_GAUSS3_AHI_{i}{j}"] = h
            c[f"CL_GAUSS3_ALO_{i}{j}"] = float(A[i][j] - Decimal(h))
    for i in range(3):
        h = float(b[i])
        c[f"CL_GAUSS3_BHI_{i}"] = h
        c[f"CL_GAUSS3_BLO_{i}"] = float(b[i] - Decimal(h))
    # Taylor coefficients of sin (x^3 .. x^17) and cos (x^2 .. x^16) about 0, and of
    # log(1+f) = f - f^2/2 + s (f^2/2 + R(s^2)), s = f / (2 + f), R(z) = sum_i 2 z^i / (2 i + 1) (the atanh series)
    for n in range(1, 9):
        c[f"CL_SIN_T{2 * n + 1}"] = float(Decimal((-1) ** n) / math.factorial(2 * n + 1))
        c[f"CL_COS_T{2 * n}"] = float(Decimal((-1) ** n) / math.factorial(2 * n))
    for i in range(1, 10):
        c[f"CL_LOG_T{i}"] = float(Decimal(2) / (2 * i + 1))
    c["CL_SQRT2"] = float(Decimal(2).sqrt())
    # exp: 1 / ln 2 for k = rint(x / ln 2), the reduction x - k ln 2 by the split ln 2 above, and the Taylor
    # coefficients 1 / n! of exp on |r| <= ln 2 / 2 (n = 2 .. 13; the terms 1 and r are exact)
    c["CL_INV_LN2"] = float(1 / ln2)
    for n in range(2, 14):
        c[f"CL_EXP_T{n}"] = float(Decimal(1) / math.factorial(n))
    # atan: atan(k / 16), k = 0 .. 16, as a correctly rounded head and the rounded remainder, for
    # atan(z) = atan(c) + atan((z - c) / (1 + z c)) with c = k / 16 nearest to z in [0, 1]; the Taylor
    # coefficients (-1)^n / (2 n + 1) of atan(u) (n = 1 .. 6) on |u| <= 1 / 32; pi and pi / 2 split in two
    for k in range(17):
        a = _arctan_frac(k, 16)
        c[f"CL_ATAN_HI_{k}"] = float(a)
        c[f"CL_ATAN_LO_{k}"] = float(a - Decimal(c[f"CL_ATAN_HI_{k}"]))
    for n in range(1, 7):
        c[f"CL_ATAN_T{2 * n + 1}"] = float(Decimal((-1) ** n) / (2 * n + 1))
    c["CL_PI_HI"] = float(pi)
    c["CL_PI_LO"] = float(pi - Decimal(c["CL_PI_HI"]))
    return c


def render(c: dict[str, float], guard: str, what: str) -> str:
    lines = [f"/* {what}", " * Generated by chaos_b200/csrc/derive_constants.py from the mathematical definitions (do not edit). */",
             f"#ifndef {guard}", f"#define {guard}", ""]
    for k, v in c.items():
        lines.append(f"#define {k} ({v.hex()})")
    lines += ["", f"#endif /* {guard} */", ""]
    return "\n".join(lines)


def main() -> None:
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    c = derive()
    targets = {
        os.path.join(root, "chaos_b200", "csrc", "cl_constants.h"): ("CL_CONSTANTS_H", "Constants of the B200 engine."),
        os.path.join(root, "oracle", "oracle_constants.hpp"): ("ORACLE_CONSTANTS_HPP", "Constants of the CPU oracle."),
    }
    for path, (guard, what) in targets.items():
        with open(path, "w") as f:
            f.write(render(c, guard, what))
        print("wrote", path, file=sys.stderr)


if __name__ == "__main__":
    main()
