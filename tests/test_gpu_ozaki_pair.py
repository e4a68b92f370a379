"""Ozaki products of at least 256 x 256 run on CTA pairs (256 x 256 tiles on
two SMs), and large products fold their levels in a kernel of their own
after the GEMM instead of in its epilogue. The INT32 level sums are exact
and every fold is the same FP64 arithmetic in the same order, so every FP64
routine must give bit-identical results with the pair engine on and off and
with either fold. The choices are read once per process (TB_OZ_PAIR,
TB_OZ_FOLD), so each setting runs in its own subprocess. The cases cover ragged edges (rows and columns past a
pair tile's halves), both triangles, transposes, K chunks with accumulation,
SYR2K's shifted K blocks, triangular K ranges (TRMM, TRSM leaves), rows
whose fold scales leave the normal double range, and the raw INT32 level
sums."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import ctypes, hashlib, sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
import TensorBLAS as TB
lib = TB.lib
P, L, D, I, Ch = ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_int, ctypes.c_char
lib.tb_dsyrk_ozaki.argtypes = [Ch, Ch, L, L, D, P, L, D, P, L, I]
lib.tb_dsyr2k_ozaki.argtypes = [Ch, Ch, L, L, D, P, L, P, L, D, P, L, I]
lib.tb_dtrmm_ozaki.argtypes = [Ch, L, L, D, P, L, P, L, P, L, I]
lib.tb_dtrsm_ozaki.argtypes = [Ch, L, L, P, L, P, L, L, I]
lib.tb_ozaki_level_product.argtypes = [L, L, P, L, I, I, P, L]
g = np.random.Generator(np.random.PCG64(23))

def dev(x):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x, np.float64).T)).cuda()

def wide(r, c, phi=1.0):
    return g.standard_normal((r, c)) * np.exp(phi * g.standard_normal((r, c)))

def ok(s):
    assert s == 0, (s, lib.tb_last_error())

out = []
def digest(t):
    TB.synchronize()
    x = t.cpu().numpy()
    out.append(hashlib.sha1(x.tobytes()).hexdigest())

for uplo, trans, n, k, S in [(b"L", b"N", 600, 700, 8), (b"U", b"T", 520, 300, 11), (b"L", b"N", 256, 10000, 14)]:
    A = wide(n, k) if trans == b"N" else wide(k, n)
    dA, dC = dev(A), dev(g.standard_normal((n, n)))
    ok(lib.tb_dsyrk_ozaki(uplo, trans, n, k, -0.75, dA.data_ptr(), A.shape[0], 0.5, dC.data_ptr(), n, S))
    digest(dC)
# rows of very different magnitudes: some fold scales leave the normal range
n, k = 300, 200
A = wide(n, k, 0.5) * np.exp2(g.integers(-600, 500, n)).reshape(n, 1)
dA, dC = dev(A), dev(np.zeros((n, n)))
ok(lib.tb_dsyrk_ozaki(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, 8))
digest(dC)
for n, k, S in [(384, 257, 10), (700, 129, 7)]:
    A, B = wide(n, k), wide(n, k)
    dA, dB, dC = dev(A), dev(B), dev(g.standard_normal((n, n)))
    ok(lib.tb_dsyr2k_ozaki(b"L", b"N", n, k, 1.25, dA.data_ptr(), n, dB.data_ptr(), n, 2.0, dC.data_ptr(), n, S))
    digest(dC)
for uplo, m, n in [(b"L", 700, 300), (b"U", 520, 600)]:
    A, B = wide(m, m), wide(m, n)
    dA, dB, dC = dev(A), dev(B), dev(np.zeros((m, n)))
    ok(lib.tb_dtrmm_ozaki(uplo, m, n, 0.5, dA.data_ptr(), m, dB.data_ptr(), m, dC.data_ptr(), m, 10))
    digest(dC)
for side, m, n, nb in [(b"R", 600, 700, 256), (b"L", 1000, 300, 512)]:
    nt = m if side == b"L" else n
    A = np.tril(g.uniform(-1, 1, (nt, nt)) / np.sqrt(nt), -1) + np.diag(g.uniform(1, 2, nt))
    dA, dB = dev(A), dev(g.uniform(-1, 1, (m, n)))
    ok(lib.tb_dtrsm_ozaki(side, m, n, dA.data_ptr(), nt, dB.data_ptr(), m, nb, 9))
    digest(dB)
n, k, S = 300, 520, 6
A = wide(n, k)
dA = dev(A)
for Lv in range(2, S + 2):
    dP = torch.zeros(n * n, dtype=torch.int32, device="cuda")
    ok(lib.tb_ozaki_level_product(n, k, dA.data_ptr(), n, S, Lv, dP.data_ptr(), n))
    digest(dP)
print(" ".join(out))
"""


def _digests(pair, fold):
    env = dict(os.environ, TB_OZ_PAIR=str(pair), TB_OZ_FOLD=fold)
    out = subprocess.run([sys.executable, "-c", SCRIPT, os.path.join(ROOT, "tensor-blas_b200", "python")], env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return out.stdout.strip().splitlines()[-1].split()


def test_engines_and_folds_are_bit_identical():
    base = _digests(0, "fused")
    assert len(base) == 16
    names = ["syrk L N", "syrk U T", "syrk K chunks", "syrk wide exponents", "syr2k", "syr2k k 129", "trmm L", "trmm U",
             "trsm R", "trsm L"]
    names += [f"level {L}" for L in range(2, 8)]
    for pair, fold in ((1, "fused"), (0, "split"), (1, "split")):
        other = _digests(pair, fold)
        diff = [nm for nm, a, b in zip(names, base, other) if a != b]
        assert not diff, (pair, fold, diff)
