"""The persistent TRSM solve (one launch for every leaf product and update of
the recursion, scheduled on the device by progress counters) gives results
bit-identical to the launch-per-product recursion: the same tiles, K ranges,
operands and epilogue roundings, applied to each output tile in the same
order. The path is chosen once per process (TB_TRSM_DAG), so each setting
runs in its own subprocess; the cases cover both sides, both precisions,
ragged leaves and strips, and the benchmark's 16384 / nb 512 solve."""
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
side, m, n, nb, prec = sys.argv[2], int(sys.argv[3]), int(sys.argv[4]), int(sys.argv[5]), int(sys.argv[6])
nt = m if side == "L" else n
g = torch.Generator(device="cuda")
g.manual_seed(nt * 7 + m + n)
L = torch.tril(torch.rand(nt, nt, device="cuda", generator=g) * 2 - 1, -1) / nt ** 0.5
L += torch.diag(torch.rand(nt, device="cuda", generator=g) + 1)
dA = L.t().contiguous()
del L
dB = torch.rand(n, m, device="cuda", generator=g) * 2 - 1   # column-major m x n
TB._bind_stream(dB)
l0 = TB.lib.tb_launch_count()
TB.strsm(side, dA, dB, m, n, nt, m, nb, prec)
TB.synchronize()
launches = TB.lib.tb_launch_count() - l0
X = dB.cpu().numpy()
assert np.all(np.isfinite(X))
print(launches, hashlib.sha1(X.tobytes()).hexdigest())
"""


def _run(dag, side, m, n, nb, prec):
    env = dict(os.environ, TB_TRSM_DAG="1" if dag else "0")
    out = subprocess.run([sys.executable, "-c", SCRIPT, os.path.join(ROOT, "tensor-blas_b200", "python"), side,
                          str(m), str(n), str(nb), str(prec)], env=env, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-3000:]
    launches, digest = out.stdout.strip().splitlines()[-1].split()
    return int(launches), digest


@pytest.mark.parametrize("side,m,n,nb,prec", [
    ("L", 2048, 3000, 512, 0),    # plain, ragged strips
    ("R", 2900, 2048, 512, 0),
    ("L", 2500, 1300, 512, 0),    # ragged last leaf (452 rows)
    ("R", 700, 2500, 256, 1),     # split
    ("L", 4096, 4096, 256, 1),
    ("L", 1536, 1000, 512, 0),    # order < 2048: the plain form runs split products
    ("L", 16384, 16384, 512, 0),  # the benchmark's solve
])
def test_persistent_solve_is_bit_identical_to_launch_per_product(side, m, n, nb, prec):
    l_dag, d_dag = _run(True, side, m, n, nb, prec)
    l_seq, d_seq = _run(False, side, m, n, nb, prec)
    print(f"{side} {m}x{n} nb={nb} prec={prec}: launches persistent {l_dag}, per-product {l_seq}")
    assert d_dag == d_seq
    assert l_dag < l_seq
