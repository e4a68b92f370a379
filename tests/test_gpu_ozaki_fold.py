"""The FP64 result of the Ozaki DSYRK is, element by element, the per-level
fold chain with one correct rounding (to nearest, ties to even) per level:

    C_1 = RN(beta C_0)            (C_1 = 0 for beta = 0: C is not read)
    C_L = RN(alpha 2^(e_i + e_j - 7L) P_L + C_(L-1)),  L = 2 .. S + 1

(P_L the exact INT32 level sums, e the row exponents), each step one fma()
while alpha 2^(e_i + e_j - 7L) is a normal double or an exact subnormal
power of two (a level whose scale lies below 2^-1074 is dropped). This test
replays the chain with exact rationals from the oracle's slices and level
products (both pinned bit-exact against the library in test_gpu_ozaki.py)
and requires bit-identical results, on a single-CTA size and on a CTA-pair
size, with rows of very different magnitudes."""
import ctypes
import math
from fractions import Fraction

import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu


def _chain(alpha, beta, c0, e_i, e_j, levels):
    """The chain as doubles; float(Fraction) rounds correctly and keeps the
    sign of a result that underflows to zero; an exact zero is -0 only when
    both addends are -0 (alpha 2^k * 0 carries alpha's sign)."""
    c = 0.0 if beta == 0.0 else float(Fraction(beta) * Fraction(c0))
    for L, p in levels:
        p = int(p)
        if p == 0 and c == 0.0:
            c = -0.0 if (math.copysign(1.0, c) < 0 and alpha < 0) else 0.0
        else:
            c = float(Fraction(alpha) * Fraction(2) ** (e_i + e_j - 7 * L) * p + Fraction(c))
    return c


@pytest.mark.parametrize("n,k,S,alpha,beta", [(96, 80, 6, -0.75, 0.5), (288, 64, 5, 1.0, 0.0)])
def test_dsyrk_fold_is_correctly_rounded_per_level(tblas, n, k, S, alpha, beta):
    lib = tblas.lib
    P, L_ = ctypes.c_void_p, ctypes.c_long
    lib.tb_dsyrk_ozaki.argtypes = [ctypes.c_char, ctypes.c_char, L_, L_, ctypes.c_double, P, L_, ctypes.c_double, P,
                                   L_, ctypes.c_int]
    g = np.random.Generator(np.random.PCG64(n + k))
    A = g.standard_normal((n, k)) * np.exp(g.standard_normal((n, k)))
    A[::17] *= 2.0 ** -300
    A[5::23] *= 2.0 ** 300
    C0 = g.standard_normal((n, n))
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dC = torch.from_numpy(np.ascontiguousarray(C0.T)).cuda()
    tblas._check(lib.tb_dsyrk_ozaki(b"L", b"N", n, k, alpha, dA.data_ptr(), n, beta, dC.data_ptr(), n, S))
    tblas.synchronize()
    C = dC.cpu().numpy().T
    Q, e = orc.ozaki_slices(A, S)
    Pl = [(L, orc.ozaki_level_product(Q, L)) for L in range(2, S + 2)]
    r, c = np.tril_indices(n)
    if r.size > 6000:
        pick = g.choice(r.size, 6000, replace=False)
        r, c = r[pick], c[pick]
    bad = []
    for i, j in zip(r.tolist(), c.tolist()):
        want = _chain(alpha, beta, C0[i, j], int(e[i]), int(e[j]), [(L, p[i, j]) for L, p in Pl])
        got = float(C[i, j])
        if np.float64(got).view(np.uint64) != np.float64(want).view(np.uint64):
            bad.append((i, j, got, want))
    assert not bad, bad[:5]
    assert np.array_equal(np.triu(C, 1), np.triu(C0, 1))
