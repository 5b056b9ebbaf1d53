"""Constants of the table-driven FP64 exp in common.cuh (exp_tab).

The method is Tang's ("Table-driven implementation of the exponential
function in IEEE floating-point arithmetic", ACM TOMS 15(2), 1989), with 64
table entries: exp(s) = 2^m 2^(j/64) exp(r), k = rint(s 64 / ln 2) = 64 m + j,
r = s - k ln2/64 in [-ln2/128, ln2/128].  This script prints

  * T[j] = 2^(j/64), j = 0..63, correctly rounded to double;
  * ln2/64 split as L_hi (its leading 32 bits, so k L_hi is exact for
    |k| < 2^21) + L_lo;
  * 64 / ln 2,

computed with 60-digit decimal arithmetic.  exp(r) - 1 = r + r^2 (1/2 + r/6 +
r^2/24 + r^3/120 + r^4/720) is the Taylor polynomial (truncation < 3.6e-17
for |r| <= ln2/128), so it needs no fitted constants.

    python exp_table_gen.py
"""
import decimal
import struct

D = decimal.Decimal
decimal.getcontext().prec = 60


def to_double(x: D) -> float:
    # correctly rounded: Python's float() of a Decimal rounds to nearest
    return float(x)


def hexd(v: float) -> str:
    return "0x%016x" % struct.unpack("<Q", struct.pack("<d", v))[0]


def main() -> None:
    ln2 = D(2).ln()
    tab = [to_double((ln2 * j / 64).exp()) for j in range(64)]
    l = ln2 / 64
    lf = to_double(l)
    bits = struct.unpack("<Q", struct.pack("<d", lf))[0]
    l_hi = struct.unpack("<d", struct.pack("<Q", bits & ~((1 << 21) - 1)))[0]  # 53 - 21 = 32 bits
    l_lo = to_double(l - D(l_hi))
    inv = to_double(64 / ln2)
    print("T[j] = 2^(j/64):")
    for j in range(0, 64, 2):
        print(f"  {tab[j]!r}, {tab[j + 1]!r},")
    print(f"L_hi = {l_hi!r} ({hexd(l_hi)})")
    print(f"L_lo = {l_lo!r} ({hexd(l_lo)})")
    print(f"64/ln2 = {inv!r}")


if __name__ == "__main__":
    main()
