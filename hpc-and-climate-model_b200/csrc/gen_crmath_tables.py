"""Generate uw_crmath_tables.h: the constants of the correctly rounded exp/log/pow of uw_math.h.

Every value is computed here from its mathematical definition with mpmath at 400 bits and rounded
to double with Python's correctly rounded int/int division (Fraction -> float):

  exp:  T[j] = 2^(j/64), j = 0..63, as a double-double (hi = RN(T), lo = RN(T - hi));
        ln2/64 split in three parts C1 + C2 + C3, C1 and C2 with at most 35 significant bits (so
        that k*C1 and k*C2 are exact for |k| < 2^17), C3 = RN(ln2/64 - C1 - C2); 64/ln2 rounded.
  log:  for m in [sqrt(1/2), sqrt(2)) the bin i = floor(128 m) - 90 (0..91) gets a reciprocal
        INVC[i] with at most 7 significant bits close to 1/(bin centre) (exactly 1 for the two bins
        that touch m = 1), and LOGC[i] = -log(INVC[i]) as a double-double.  With 7-bit INVC the
        product m * INVC is a multiple of 2^-59, so t = fma(m, INVC, -1) is exact whenever
        |t| < 2^-6; the script checks that bound over every bin.
        ln2 split as LN2H (42 significant bits, so e * LN2H is exact for |e| < 2^11) + LN2L.
  Taylor coefficients 1/n! and 1/n as double-doubles where they are not exact.

Run: python gen_crmath_tables.py  (rewrites uw_crmath_tables.h next to this script).
"""
import os
from fractions import Fraction

import mpmath

mpmath.mp.prec = 400
HERE = os.path.dirname(os.path.abspath(__file__))


def frac(x):
    """Exact rational value of an mpmath number."""
    sign, m, e, _ = mpmath.mpf(x)._mpf_
    m = -int(m) if sign else int(m)
    return Fraction(m) * (Fraction(2) ** int(e)) if e >= 0 else Fraction(m, 2 ** int(-e))


def rn(q):
    """Round a rational to the nearest double (ties to even)."""
    return float(q) if q.denominator != 1 else float(q.numerator)


def dd(x):
    q = frac(x)
    hi = rn(q)
    lo = rn(q - Fraction(hi))
    return hi, lo


def round_bits(q, bits):
    """Round a nonzero rational to `bits` significant bits (nearest)."""
    if q < 0:
        return -round_bits(-q, bits)
    assert q > 0
    e = 0
    while q >= 2:
        q /= 2
        e += 1
    while q < 1:
        q *= 2
        e -= 1
    s = round(q * 2 ** (bits - 1))
    return Fraction(s, 2 ** (bits - 1)) * (Fraction(2) ** e)


def sig_bits(v):
    q = Fraction(v)
    n = q.numerator
    d = q.denominator
    while n % 2 == 0 and n:
        n //= 2
    return n.bit_length()


def fmt(v):
    return repr(float(v)) if v != 0 else "0.0"


def main():
    ln2 = mpmath.log(2)
    L = frac(ln2 / 64)
    c1 = round_bits(L, 35)
    c2 = round_bits(L - c1, 35)
    c3 = rn(L - c1 - c2)
    assert sig_bits(float(c1)) <= 35 and sig_bits(float(c2)) <= 35
    assert Fraction(float(c1)) == c1 and Fraction(float(c2)) == c2
    invl = rn(1 / L)

    tab_exp = [dd(mpmath.mpf(2) ** (mpmath.mpf(j) / 64)) for j in range(64)]

    ln2q = frac(ln2)
    ln2h = round_bits(ln2q, 42)
    ln2l = rn(ln2q - ln2h)
    assert Fraction(float(ln2h)) == ln2h

    lo_m = frac(mpmath.sqrt(mpmath.mpf(1) / 2))
    # frexp's mantissa below RN(sqrt(1/2)) is doubled: m < 2 RN(sqrt(1/2)), a little above sqrt(2)
    hi_m = 2 * Fraction(rn(lo_m))
    invc, logc = [], []
    tmax = Fraction(0)
    for i in range(92):
        a = Fraction(90 + i, 128)
        b = Fraction(91 + i, 128)
        a = max(a, lo_m)
        b = min(b, hi_m)
        if i in (37, 38):          # bins [127/128, 1) and [1, 129/128)
            r = Fraction(1)
        else:
            r = round_bits(2 / (a + b), 7)
        # largest |m r - 1| over the bin (endpoints; linear in m)
        t = max(abs(a * r - 1), abs(b * r - 1))
        assert t < Fraction(1, 64), (i, float(t))
        tmax = max(tmax, t)
        invc.append(float(r))
        assert Fraction(float(r)) == r and sig_bits(float(r)) <= 7
        logc.append(dd(-mpmath.log(mpmath.mpf(float(r)))))

    # 1/n! (exp) and (-1)^(n+1)/n (log1p) as double-doubles
    fact = [dd(mpmath.mpf(1) / mpmath.factorial(n)) for n in range(0, 14)]
    l1p = [dd(mpmath.mpf((-1) ** (n + 1)) / n) if n else (0.0, 0.0) for n in range(0, 18)]

    out = []
    w = out.append
    w("// uw_crmath_tables.h -- generated by gen_crmath_tables.py from the mathematical definitions")
    w("// (mpmath, 400 bits, rounded to nearest double).  Do not edit.")
    w("#pragma once")
    w("")
    w("#define UW_CR_INVL %s    /* RN(64 / ln2) */" % fmt(invl))
    w("#define UW_CR_C1 %s    /* ln2/64, 35 significant bits */" % fmt(float(c1)))
    w("#define UW_CR_C2 %s    /* next 35 bits */" % fmt(float(c2)))
    w("#define UW_CR_C3 %s    /* RN(ln2/64 - C1 - C2) */" % fmt(c3))
    w("#define UW_CR_LN2H %s    /* ln2, 42 significant bits */" % fmt(float(ln2h)))
    w("#define UW_CR_LN2L %s    /* RN(ln2 - LN2H) */" % fmt(ln2l))
    w("#define UW_CR_SQRTH %s    /* RN(sqrt(1/2)) */" % fmt(rn(lo_m)))
    w("// largest |t| = |m INVC - 1| over the log bins: %.6g (< 2^-6)" % float(tmax))
    w("")
    for n in range(3, 14):
        h, l = fact[n]
        w("#define UW_CR_F%d_H %s    /* 1/%d! */" % (n, fmt(h), n))
        w("#define UW_CR_F%d_L %s" % (n, fmt(l)))
    for n in range(2, 18):
        h, l = l1p[n]
        w("#define UW_CR_L%d_H %s    /* (-1)^(n+1)/n, n = %d */" % (n, fmt(h), n))
        w("#define UW_CR_L%d_L %s" % (n, fmt(l)))
    w("")
    w("// 2^(j/64) = UW_CR_EXPT[2j] + UW_CR_EXPT[2j+1]")
    w("#define UW_CR_EXPT_INIT { \\")
    for j, (h, l) in enumerate(tab_exp):
        w("    %s, %s,%s \\" % (fmt(h), fmt(l), "" if j < 63 else ""))
    w("}")
    w("// bin i: INVC, -log(INVC) hi, lo")
    w("#define UW_CR_LOGT_INIT { \\")
    for i in range(92):
        w("    %s, %s, %s, \\" % (fmt(invc[i]), fmt(logc[i][0]), fmt(logc[i][1])))
    w("}")
    w("")
    with open(os.path.join(HERE, "uw_crmath_tables.h"), "w") as f:
        f.write("\n".join(out))


if __name__ == "__main__":
    main()
