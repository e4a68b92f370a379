"""Lower SYRKs of order >= 8192 convert A in row bands (four by default) and
launch each band's tiles as soon as its conversion lands, on two auxiliary
streams; the tiles, their K ranges and FP32 sums are those of the single
launch, so the result must be bit-identical to it (TB_SYRK_PARTS sets the
band count, 1 keeps one conversion and one launch; read once per process,
so each setting runs in a subprocess). Cases: both precisions, 'N' and 'T',
a ragged order, a beta != 0 and other band counts."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import hashlib, sys, torch
sys.path.insert(0, sys.argv[1])
import TensorBLAS as TB
trans, n, k, prec, beta = sys.argv[2], int(sys.argv[3]), int(sys.argv[4]), int(sys.argv[5]), float(sys.argv[6])
g = torch.Generator(device="cuda")
g.manual_seed(n + k)
rows = k if trans == "T" else n
A = torch.rand(k if trans == "N" else n, rows, device="cuda", generator=g) * 2 - 1   # column-major op storage
C = torch.rand(n, n, device="cuda", generator=g) * 2 - 1
TB._bind_stream(A)
TB._check(TB.lib.tb_ssyrk(b"L", trans.encode(), n, k, 1.5, A.data_ptr(), rows, beta, C.data_ptr(), n, 256, prec))
TB.synchronize()
print(hashlib.sha1(C.cpu().numpy().tobytes()).hexdigest())
"""


def _digest(parts, trans, n, k, prec, beta, **extra):
    env = dict(os.environ, TB_SYRK_PARTS=parts, **extra)
    out = subprocess.run([sys.executable, "-c", SCRIPT, os.path.join(ROOT, "tensor-blas_b200", "python"), trans,
                          str(n), str(k), str(prec), str(beta)], env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return out.stdout.strip().splitlines()[-1]


@pytest.mark.parametrize("trans,n,k,prec,beta", [("N", 8192, 2048, 0, 0.0), ("N", 8448, 1100, 0, 0.5),
                                                 ("T", 8192, 1536, 0, 0.0), ("N", 8192, 1088, 1, 0.0)])
def test_banded_syrk_is_bit_identical_to_single_launch(trans, n, k, prec, beta):
    assert _digest("1", trans, n, k, prec, beta) == _digest("4", trans, n, k, prec, beta)


def test_band_count_does_not_change_the_bits():
    ref = _digest("1", "N", 8448, 1100, 0, 0.5)
    for parts in ("2", "7", "16"):
        assert _digest(parts, "N", 8448, 1100, 0, 0.5) == ref, parts


@pytest.mark.parametrize("trans,n,k", [("N", 8448, 1100), ("T", 4096, 3000)])
def test_direct_store_epilogue_is_bit_identical(trans, n, k):
    """beta = 0 CTA-pair launches store from registers with a seventh operand
    stage (TB_GEMM_PAIR_DIRECT=0 keeps the staged TMA epilogue): same bits."""
    assert _digest("1", trans, n, k, 0, 0.0, TB_GEMM_PAIR_DIRECT="0") == _digest("1", trans, n, k, 0, 0.0)


def test_pair_and_single_cta_engines_give_the_same_bits():
    """Large plain launches on CTA pairs (256 x 256 tiles, the default) or on
    single CTAs (128 x 256, TB_GEMM_PAIR=0): each element is the same
    K-ordered FP32 accumulation of the same FP16 products."""
    assert _digest("1", "N", 4096, 3000, 0, 0.5, TB_GEMM_PAIR="0") == _digest("1", "N", 4096, 3000, 0, 0.5)
