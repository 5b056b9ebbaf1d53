"""The two-MMA split-FP16 operand layout of the symmetric tensor-core kernel
(csrc/matvec_symtc.cu, k1t_pack16x2_kernel), checked on the host.

For embeddings of at most 10 padded dimensions the three split-FP16 products
H H' + Hs L' + L Hs' are computed as V0 W0 + V1 W1 with
V0 = [H | Hs_0..Hs_P-1], V1 = [Hs_P..Hs_DP-1 | L | 0], W0 = [H' | L'_0..L'_P-1]
and W1 = [L'_P..L'_DP-1 | Hs' | 0], P = min(16 - DP, DP).  The same FP16
values enter the same products, so in exact arithmetic the two forms agree to
the last bit; this test restates the index mapping of the pack kernel and
checks that identity for every DP the format accepts.  The GPU tests check
the kernel itself against the float64 oracle.
"""

from fractions import Fraction

import numpy as np
import pytest


def _split(v):
    h = v.astype(np.float16)
    lo = ((v - h.astype(np.float32)) * np.float32(4096.0)).astype(np.float16)
    hs = (h.astype(np.float32) / np.float32(4096.0)).astype(np.float16)
    return h, lo, hs


def _variants(h, lo, hs, dp, row):
    """The pack kernel's four 16-wide variants for one side."""
    p = min(16 - dp, dp)
    rest = dp - p
    v0 = np.zeros(16, np.float16)
    v1 = np.zeros(16, np.float16)
    first, second = (hs, lo) if row else (lo, hs)
    for k in range(16):
        if k < dp:
            v0[k] = h[k]
        elif k - dp < p:
            v0[k] = first[k - dp]
        if k < rest:
            v1[k] = first[p + k]
        elif k - rest < dp:
            v1[k] = second[k - rest]
    return v0, v1


def _dot(a, b):
    return sum(Fraction(float(x)) * Fraction(float(y)) for x, y in zip(a, b))


@pytest.mark.parametrize("dp", [2, 4, 6, 8, 10])
def test_two_mma_layout_gives_the_three_products(dp):
    rng = np.random.default_rng(dp)
    for _ in range(20):
        a = np.zeros(16, np.float32)
        b = np.zeros(16, np.float32)
        a[:dp] = rng.standard_normal(dp).astype(np.float32) * 2
        b[:dp] = rng.standard_normal(dp).astype(np.float32) * 2
        ha, la, hsa = _split(a * np.float32(1.4426950408889634))  # row side: log2 e folded in
        hb, lb, hsb = _split(b)
        three = _dot(ha, hb) + _dot(hsa, lb) + _dot(la, hsb)
        v0, v1 = _variants(ha, la, hsa, dp, row=True)
        w0, w1 = _variants(hb, lb, hsb, dp, row=False)
        assert _dot(v0, w0) + _dot(v1, w1) == three
