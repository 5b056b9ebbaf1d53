"""The table-driven FP64 exp of the FP64 operator kernels (csrc/common.cuh,
exp_tab), checked on the host.

* The 64-entry table of 2^(j/64) and the reduction constants compiled into
  the kernels are the correctly rounded values (recomputed here with 60-digit
  decimal arithmetic, as csrc/exp_table_gen.py does).
* The algorithm, restated step by step with every fused multiply-add rounded
  once (exact rational arithmetic), stays within 1.5 ulp of exp on random
  arguments over the range the kernels use, and gives 1 at 0.

The GPU tests check the same kernels against the float64 oracle to 1e-12.
"""

import decimal
import math
import re
import struct
from fractions import Fraction
from pathlib import Path

import numpy as np

CSRC = Path(__file__).resolve().parents[1] / "learning-based-attention-kernel-regression_b200" / "csrc"


def _header():
    return (CSRC / "common.cuh").read_text()


def _table():
    src = _header()
    body = re.search(r"c_exp2_64\[64\]\s*=\s*\{([^}]*)\}", src).group(1)
    vals = [float(t) for t in body.replace("\n", " ").split(",") if t.strip()]
    assert len(vals) == 64
    return vals


def _const(name):
    m = re.search(r"constexpr double %s = ([0-9.eE+-]+);" % name, _header())
    return float(m.group(1))


def test_table_and_constants_are_correctly_rounded():
    decimal.getcontext().prec = 60
    ln2 = decimal.Decimal(2).ln()
    for j, v in enumerate(_table()):
        assert v == float((ln2 * j / 64).exp())
    assert _const("kInvL") == float(64 / ln2)
    hi, lo = _const("kLhi"), _const("kLlo")
    # kLhi keeps the leading 32 bits of ln2/64 (k * kLhi exact for |k| < 2^21)
    bits = struct.unpack("<Q", struct.pack("<d", hi))[0]
    assert bits & ((1 << 21) - 1) == 0
    assert float(ln2 / 64 - decimal.Decimal(hi)) == lo


def _fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _exp_tab(s, tab, inv_l, l_hi, l_lo):
    rnd = 6755399441055744.0
    t = _fma(s, inv_l, rnd)
    kd = t - rnd
    lo32 = struct.unpack("<Q", struct.pack("<d", t))[0] & 0xFFFFFFFF
    k = lo32 - (1 << 32) if lo32 >= (1 << 31) else lo32
    r = _fma(-kd, l_hi, s)
    r = _fma(-kd, l_lo, r)
    q = _fma(r, 1.0 / 120.0, 1.0 / 24.0)
    q = _fma(q, r, 1.0 / 6.0)
    q = _fma(q, r, 0.5)
    p = _fma(r * r, q, r)
    tj = tab[k & 63]
    m = max(-1022, min(1023, k >> 6))
    scale = struct.unpack("<d", struct.pack("<Q", (m + 1023) << 52))[0]
    return _fma(tj, p, tj) * scale


def test_algorithm_error_bound():
    tab = _table()
    consts = (_const("kInvL"), _const("kLhi"), _const("kLlo"))
    rng = np.random.default_rng(0)
    samples = np.concatenate([rng.uniform(-80, 80, 1500), rng.uniform(-700, 700, 500),
                              rng.uniform(-1e-3, 1e-3, 200)])
    worst = 0.0
    for s in samples:
        s = float(s)
        got = _exp_tab(s, tab, *consts)
        ref = math.exp(s)
        ulp = math.ulp(ref)
        worst = max(worst, abs(got - ref) / ulp)
    assert worst <= 1.5, worst
    assert _exp_tab(0.0, tab, *consts) == 1.0
