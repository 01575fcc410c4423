"""Writes the constants of vh_crmath.cuh: ln 2 split into three doubles (the
first with 33 significant bits, so that k * LN2_1 is exact for |k| < 2^20),
1 / ln 2 rounded to nearest, and 1/n! (n = 2..11) as double-double pairs.
Exact rational arithmetic (fractions) and a 60-digit decimal ln 2
(decimal.Decimal.ln); run it to check the literals in the header:

    python vhlle_b200/csrc/gen_crmath_consts.py
"""
import decimal
import math
from fractions import Fraction

decimal.getcontext().prec = 80
LN2 = Fraction(decimal.Decimal(2).ln())


def rn(q: Fraction) -> float:
    """q rounded to the nearest double (ties to even), via float(Fraction)."""
    return float(q)


def trunc_bits(q: Fraction, bits: int) -> float:
    """q > 0 truncated to `bits` significant bits (a double)."""
    exp = math.frexp(float(q))[1]
    scale = Fraction(2) ** (bits - exp)
    return float(Fraction(int(q * scale)) / scale)


def main():
    l1 = trunc_bits(LN2, 33)
    r = LN2 - Fraction(l1)
    l2 = rn(r)
    r -= Fraction(l2)
    l3 = rn(r)
    print("LN2_1 = %s  // %r" % (l1.hex(), l1))
    print("LN2_2 = %s  // %r" % (l2.hex(), l2))
    print("LN2_3 = %s  // %r" % (l3.hex(), l3))
    print("INV_LN2 = %s" % rn(1 / LN2).hex())
    f = Fraction(1)
    for n in range(1, 12):
        f /= n
        hi = rn(f)
        lo = rn(f - Fraction(hi))
        print("INV_FACT[%d] = {%s, %s}" % (n, hi.hex(), lo.hex()))


if __name__ == "__main__":
    main()
