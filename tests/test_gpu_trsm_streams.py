"""On the launch-per-product path (TB_TRSM_DAG=0), plain TRSMs with at least
4096 independent columns (left) or rows (right) can be solved in parts (up
to four, TB_TRSM_STREAMS; one by default) on as many streams; each column's
(row's) arithmetic is the same either way, so the result must be
bit-identical to the one-stream solve. The part count is read once per process (TB_TRSM_STREAMS), so each
setting runs in its own subprocess."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import hashlib, sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
import TensorBLAS as TB
side, m, n = sys.argv[2], int(sys.argv[3]), int(sys.argv[4])
g = np.random.Generator(np.random.PCG64(17))
nt = m if side == "L" else n
A = (np.tril(g.uniform(-1, 1, (nt, nt)) / np.sqrt(nt), -1) + np.diag(g.uniform(1, 2, nt))).astype(np.float32)
B = g.uniform(-1, 1, (m, n)).astype(np.float32)
dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
TB.strsm(side, dA, dB, m, n, nt, m, 512, TB.PLAIN)
TB.synchronize()
X = dB.cpu().numpy()
assert np.all(np.isfinite(X))
print(hashlib.sha1(X.tobytes()).hexdigest())
"""


def _digest(streams, side, m, n):
    env = dict(os.environ, TB_TRSM_STREAMS=str(streams), TB_TRSM_DAG="0")
    out = subprocess.run([sys.executable, "-c", SCRIPT, os.path.join(ROOT, "tensor-blas_b200", "python"), side,
                          str(m), str(n)], env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return out.stdout.strip().splitlines()[-1]


@pytest.mark.parametrize("side,m,n", [("L", 2048, 4608), ("R", 4608, 2048)])
def test_two_stream_solve_is_bit_identical(side, m, n):
    assert _digest(1, side, m, n) == _digest(2, side, m, n)


@pytest.mark.parametrize("side,m,n", [("L", 1536, 5000), ("R", 5000, 1536)])
def test_three_and_four_part_solves_are_bit_identical(side, m, n):
    ref = _digest(1, side, m, n)
    assert _digest(3, side, m, n) == ref
    assert _digest(4, side, m, n) == ref
