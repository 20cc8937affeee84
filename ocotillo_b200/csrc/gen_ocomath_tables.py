#!/usr/bin/env python3
"""Generate ``ocomath_tables.h``: the constant tables of the shared exp/log core.

The tables are evaluated with Python's ``decimal`` module at 80 significant digits
(correctly rounded exp/ln at that precision) and split into double-double pairs
(hi = RN(v), lo = RN(v - hi)).  Run from anywhere:

    python ocotillo_b200/csrc/gen_ocomath_tables.py > ocotillo_b200/csrc/ocomath_tables.h

Method references (the algorithms the tables serve):
  * P. T. P. Tang, "Table-driven implementation of the exponential function in
    IEEE floating-point arithmetic", ACM TOMS 15(2), 1989.
  * P. T. P. Tang, "Table-driven implementation of the logarithm function in IEEE
    floating-point arithmetic", ACM TOMS 16(4), 1990.
"""
from decimal import Decimal, getcontext
from fractions import Fraction
import math

getcontext().prec = 80

EXP_N = 128            # exp table: 2^(j/128), j = 0..127
EXP_FAST_N = 1024      # fast exp phase: 2^(j/1024), j = 0..1023
LOG_N = 128            # log table: F = 1 + j/128, j = LOG_JMIN..LOG_JMAX
LOG_JMIN, LOG_JMAX = -32, 64

LN2 = Decimal(2).ln()
LN10 = Decimal(10).ln()
LOG10E = 1 / LN10


def rn(d: Decimal) -> float:
    """Round a Decimal to the nearest double (Python's float(Decimal) is correctly rounded)."""
    return float(d)


def dd(d: Decimal):
    hi = rn(d)
    lo = rn(d - Decimal(hi))
    return hi, lo


def trunc_bits(d: Decimal, bits: int) -> float:
    """Truncate a positive Decimal to ``bits`` significant bits (exactly representable)."""
    f = Fraction(d)
    e = 0
    while f >= 2 ** bits:
        f /= 2
        e += 1
    while f < 2 ** (bits - 1):
        f *= 2
        e -= 1
    n = math.floor(f)
    return math.ldexp(float(n), e)


def h(x: float) -> str:
    if x == 0.0:
        return "0.0"
    return x.hex()


def emit_pairs(name, pairs, per_line=2):
    out = [f"OCO_MATH_TABLE({name}, {2 * len(pairs)}) = {{"]
    row = []
    for hi, lo in pairs:
        row.append(f"{h(hi)}, {h(lo)}")
        if len(row) == per_line:
            out.append("  " + ", ".join(row) + ",")
            row = []
    if row:
        out.append("  " + ", ".join(row) + ",")
    out.append("};")
    return "\n".join(out)


def main():
    lines = []
    lines.append("/* Generated by gen_ocomath_tables.py -- do not edit by hand.")
    lines.append(" * Double-double tables for the ocomath exp/log core (see ocomath.h). */")
    lines.append("/* Included twice by ocomath.h (host copy and device copy); no include guard. */")
    lines.append("")
    # exp: 2^(j/N) as (hi, lo)
    exp_pairs = [dd((Decimal(j) / EXP_N * LN2).exp()) for j in range(EXP_N)]
    lines.append(f"#define OCO_EXP_N {EXP_N}")
    lines.append(emit_pairs("oco_exp_tab", exp_pairs))
    lines.append("")
    # log: for j in [JMIN, JMAX]: F = 1 + j/N, log(F) and 1/F as (hi, lo)
    log_pairs, inv_pairs = [], []
    for j in range(LOG_JMIN, LOG_JMAX + 1):
        F = Decimal(1) + Decimal(j) / LOG_N
        log_pairs.append(dd(F.ln()) if j != 0 else (0.0, 0.0))
        inv_pairs.append(dd(1 / F))
    lines.append(f"#define OCO_LOG_N {LOG_N}")
    lines.append(f"#define OCO_LOG_JMIN ({LOG_JMIN})")
    lines.append(f"#define OCO_LOG_JMAX ({LOG_JMAX})")
    lines.append(emit_pairs("oco_logF_tab", log_pairs))
    lines.append(emit_pairs("oco_invF_tab", inv_pairs))
    lines.append("")
    # Cody-Waite split of ln2/N for the exp reduction: L1 has 35 significant bits so that
    # k*L1 is exact for |k| < 2^18 (|x| <= 746 gives |k| <= 137,800).
    l = LN2 / EXP_N
    L1 = trunc_bits(l, 35)
    r1 = l - Decimal(L1)
    L2 = rn(r1)
    L3 = rn(r1 - Decimal(L2))
    lines.append(f"#define OCO_EXP_INVLN2N {h(rn(EXP_N / LN2))}  /* N/ln2 */")
    lines.append(f"#define OCO_EXP_L1 {h(L1)}  /* ln2/N, 35 significant bits */")
    lines.append(f"#define OCO_EXP_L2 {h(L2)}")
    lines.append(f"#define OCO_EXP_L3 {h(L3)}")
    # Fast exp phase: 2^(j/1024) as (hi, lo) and a Cody-Waite split of ln2/1024 whose head has
    # 32 significant bits, so that k*L1 is exact for |k| < 2^21 (|x| <= 746 gives |k| <= 1.11e6).
    exp_fast = [dd((Decimal(j) / EXP_FAST_N * LN2).exp()) for j in range(EXP_FAST_N)]
    lines.append(f"#define OCO_EXPF_N {EXP_FAST_N}")
    lines.append(emit_pairs("oco_expf_tab", exp_fast))
    lf = LN2 / EXP_FAST_N
    F1 = trunc_bits(lf, 32)
    rf = lf - Decimal(F1)
    F2 = rn(rf)
    F3 = rn(rf - Decimal(F2))
    lines.append(f"#define OCO_EXPF_INVLN2N {h(rn(EXP_FAST_N / LN2))}  /* 1024/ln2 */")
    lines.append(f"#define OCO_EXPF_L1 {h(F1)}  /* ln2/1024, 32 significant bits */")
    lines.append(f"#define OCO_EXPF_L2 {h(F2)}")
    lines.append(f"#define OCO_EXPF_L3 {h(F3)}")
    # ln2 for the log reconstruction: 42-bit head so that e*LN2_HI is exact for |e| < 2^11.
    LN2_HI = trunc_bits(LN2, 42)
    LN2_LO = rn(LN2 - Decimal(LN2_HI))
    lines.append(f"#define OCO_LN2_HI {h(LN2_HI)}  /* ln2, 42 significant bits */")
    lines.append(f"#define OCO_LN2_LO {h(LN2_LO)}")
    hi, lo = dd(LN10)
    lines.append(f"#define OCO_LN10_HI {h(hi)}")
    lines.append(f"#define OCO_LN10_LO {h(lo)}")
    hi, lo = dd(LOG10E)
    lines.append(f"#define OCO_LOG10E_HI {h(hi)}")
    lines.append(f"#define OCO_LOG10E_LO {h(lo)}")
    # Taylor coefficients 1/k! (exp) and 1/k (log1p), rounded to double.
    fact = 1
    for k in range(1, 10):
        fact *= k
        lines.append(f"#define OCO_EXP_C{k} {h(rn(Decimal(1) / fact))}")
    for k in range(2, 13):
        lines.append(f"#define OCO_LOG_C{k} {h(rn(Decimal(1) / k))}")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
