"""Generate ns_crmath_consts.h: binary64 constants for the correctly rounded
binary32 exp/log in ns_crmath.h.

Every constant is computed with Python's decimal module at 80 significant
digits and rounded to binary64 by float(str(...)), which rounds correctly.
Double-double constants are (hi, lo) with hi = RN(v), lo = RN(v - hi).

Run:  python neural-selection_b200/csrc/gen_crmath_consts.py
"""
from decimal import Decimal, getcontext
from pathlib import Path

getcontext().prec = 80
TWO = Decimal(2)
LN2 = TWO.ln()


def rn(v):
    return float(str(v))


def dd(v):
    hi = rn(v)
    lo = rn(v - Decimal(hi))
    return hi, lo


def split_bits(v, bits):
    """Round v to a binary64 with at most `bits` significant bits (truncated
    toward zero), so products with small integers stay exact."""
    hi = rn(v)
    m, e = __import__('math').frexp(hi)
    scale = 2 ** bits
    t = int(m * scale) / scale
    return __import__('math').ldexp(t, e)


def hx(x):
    return float.hex(x)


lines = ["/* Generated by gen_crmath_consts.py; do not edit. */",
         "#pragma once", ""]

# 2^(j/128), j = 0..127, binary64 correctly rounded.
vals = [rn(TWO ** (Decimal(j) / 128)) for j in range(128)]
lines.append("#define NSX_EXP2_128_TABLE \\")
for i in range(0, 128, 4):
    chunk = ", ".join(hx(v) for v in vals[i:i + 4])
    sep = ", \\" if i + 4 < 128 else ""
    lines.append("    " + chunk + sep)
lines.append("")

inv = rn(Decimal(128) / LN2)
lines.append(f"#define NSX_INV_LN2_128 {hx(inv)}")
h, l = dd(LN2 / 128)
lines.append(f"#define NSX_LN2_128_HI {hx(h)}")
lines.append(f"#define NSX_LN2_128_LO {hx(l)}")
lines.append(f"#define NSX_INV_LN2 {hx(rn(1 / LN2))}")
# ln2 as a sum of three doubles whose first two have <= 45 significant
# bits, so m*A and m*B are exact for |m| < 2^8.
a = split_bits(LN2, 45)
rest = LN2 - Decimal(a)
b = split_bits(rest, 45)
c = rn(rest - Decimal(b))
lines.append(f"#define NSX_LN2_A {hx(a)}")
lines.append(f"#define NSX_LN2_B {hx(b)}")
lines.append(f"#define NSX_LN2_C {hx(c)}")
# ln2 split for log: HI has 45 bits so e*HI is exact for |e| < 2^8.
lhi = split_bits(LN2, 45)
llo = rn(LN2 - Decimal(lhi))
lines.append(f"#define NSX_LN2_LOG_HI {hx(lhi)}")
lines.append(f"#define NSX_LN2_LOG_LO {hx(llo)}")
lines.append("")

# 1/n! for n = 0..24 as double-double (exp slow path).
fact = Decimal(1)
lines.append("#define NSX_INV_FACT_DD \\")
ents = []
for n in range(25):
    if n:
        fact *= n
    h, l = dd(Decimal(1) / fact)
    ents.append(f"{hx(h)}, {hx(l)}")
for i, e in enumerate(ents):
    lines.append("    " + e + (", \\" if i + 1 < len(ents) else ""))
lines.append("#define NSX_INV_FACT_COUNT 25")
lines.append("")

# 1/(2n+1) for n = 0..23 as double-double (log slow path).
lines.append("#define NSX_INV_ODD_DD \\")
ents = []
for n in range(24):
    h, l = dd(Decimal(1) / Decimal(2 * n + 1))
    ents.append(f"{hx(h)}, {hx(l)}")
for i, e in enumerate(ents):
    lines.append("    " + e + (", \\" if i + 1 < len(ents) else ""))
lines.append("#define NSX_INV_ODD_COUNT 24")
lines.append("")

# sqrt(2) as binary64 (log argument reduction threshold; exactness is not
# required, only a fixed comparison constant).
lines.append(f"#define NSX_SQRT2 {hx(rn(TWO.sqrt()))}")

# ---- binary32 float-float fast path of exp ----
import struct


def rnf(v):
    """Round a Decimal to binary32 (via the correctly rounded binary64, then
    exactly re-rounded with ties-to-even on the 24-bit significand)."""
    d = Decimal(v)
    if d == 0:
        return 0.0
    # exact binary32 rounding of an arbitrary decimal
    import math
    sign = -1 if d < 0 else 1
    a = abs(d)
    e = int(math.floor(float(a.ln() / LN2)))
    while Decimal(2) ** e > a:
        e -= 1
    while Decimal(2) ** (e + 1) <= a:
        e += 1
    scale = Decimal(2) ** (23 - e)
    m = a * scale
    mi = int(m)
    frac = m - mi
    if frac > Decimal("0.5") or (frac == Decimal("0.5") and mi % 2 == 1):
        mi += 1
    return sign * float(Decimal(mi) / scale)


def hxf(x):
    return float.hex(x) + "f"


tabf = []
for j in range(128):
    v = TWO ** (Decimal(j) / 128)
    hi = rnf(v)
    lo = rnf(v - Decimal(hi))
    tabf += [hi, lo]
lines.append("/* 2^(j/128) as binary32 pairs (hi, lo), j = 0..127 */")
lines.append("#define NSX_EXP2F_128_TABLE \\")
for i in range(0, 256, 4):
    chunk = ", ".join(hxf(v) for v in tabf[i:i + 4])
    lines.append("    " + chunk + (", \\" if i + 4 < 256 else ""))
L = LN2 / 128
# L1: ln2/128 truncated to 10 significant bits (k*L1 exact for |k| < 2^14)
import math
m, e = math.frexp(float(L))
L1 = math.ldexp(math.floor(m * 2 ** 10) / 2 ** 10, e)
L2 = rnf(L - Decimal(L1))
L3 = rnf(L - Decimal(L1) - Decimal(L2))
lines.append(f"#define NSX_F_INV_LN2_128 {hxf(rnf(Decimal(128) / LN2))}")
lines.append(f"#define NSX_F_LN2_128_A {hxf(L1)}")
lines.append(f"#define NSX_F_LN2_128_B {hxf(L2)}")
lines.append(f"#define NSX_F_LN2_128_C {hxf(L3)}")
lines.append("")


# ---- sin / cos argument reduction ----
def pi_scaled(bits):
    """floor(pi * 2^bits) - d with 0 <= d < 2, from Machin's formula
    pi = 16 atan(1/5) - 4 atan(1/239) in integer arithmetic."""
    guard = 32
    one = 1 << (bits + guard)

    def atan_inv(n):
        total, term, k, n2 = 0, one // n, 0, n * n
        while term:
            total += term // (2 * k + 1) if k % 2 == 0 else -(term // (2 * k + 1))
            term //= n2
            k += 1
        return total
    return (16 * atan_inv(5) - 4 * atan_inv(239)) >> guard


PI_BITS = 1200
PI_INT = pi_scaled(PI_BITS)
WORDS = 12
# 2/pi = sum_i W[i] 2^(-32(i+1)): the first 32*WORDS fraction bits (2/pi < 1)
two_over_pi = (1 << (PI_BITS + 1 + 32 * WORDS)) // PI_INT
words = [(two_over_pi >> (32 * (WORDS - 1 - i))) & 0xffffffff for i in range(WORDS)]
lines.append("/* 2/pi = sum_i W[i] 2^(-32 (i + 1)) */")
lines.append("#define NSX_2OPI_WORDS \\")
lines.append("    " + ", ".join(f"0x{w:08x}u" for w in words))
lines.append(f"#define NSX_2OPI_COUNT {WORDS}")
PIO2 = Decimal(PI_INT) / (Decimal(2) ** (PI_BITS + 1))
h, l = dd(PIO2)
lines.append(f"#define NSX_PIO2_HI {hx(h)}")
lines.append(f"#define NSX_PIO2_LO {hx(l)}")
lines.append("")

out = Path(__file__).with_name("ns_crmath_consts.h")
out.write_text("\n".join(lines) + "\n")
print("wrote", out)
