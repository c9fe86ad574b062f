"""The constants of the engine and the oracle are the mathematical values, rounded once (CPU)."""
import os
import re
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "chaos_b200", "csrc"))


def _parse(path):
    out = {}
    for m in re.finditer(r"#define (CL_\w+) \(([-0-9a-fx.p+]+)\)", open(path).read()):
        out[m[1]] = float.fromhex(m[2])
    return out


def test_headers_match_derivation():
    import derive_constants as dc
    want = dc.derive()
    for p in ("chaos_b200/csrc/cl_constants.h", "oracle/oracle_constants.hpp"):
        got = _parse(os.path.join(ROOT, p))
        assert got == want, p


def test_split_properties():
    import derive_constants as dc
    from decimal import Decimal
    c = dc.derive()
    assert c["CL_PIO2_1"] == 1.5707963267948966
    # the head of ln 2 has at most 42 significant bits, so e * LN2_HI is exact for every binary64 exponent
    m, e = __import__("math").frexp(c["CL_LN2_HI"])
    assert (Decimal(m) * 2 ** 42) % 1 == 0
    # Gauss-3 weights: hi + lo is 5/18, 4/9, 5/18 to ~2^-106
    for i, v in enumerate((Decimal(5) / 18, Decimal(4) / 9, Decimal(5) / 18)):
        assert abs(Decimal(c[f"CL_GAUSS3_BHI_{i}"]) + Decimal(c[f"CL_GAUSS3_BLO_{i}"]) - v) < Decimal(2) ** -105
