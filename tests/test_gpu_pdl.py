"""TB_PDL=1 launches the GEMM engine's kernels with programmatic stream
serialization (their set-up overlaps the previous launch's last tiles, and
they wait for that launch to complete before touching global memory); the
default launches them in plain stream order. The tiles, their K order and
the sums are the same either way, so SYRK, TRSM (plain and split, left and
right), SYMM with beta != 0 and SGEMM must be bit-identical under both
settings. The switch is read once per process, so each setting runs in its
own subprocess."""
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
g = np.random.Generator(np.random.PCG64(23))
h = hashlib.sha1()
n, k = 2304, 3072
A = torch.from_numpy(g.uniform(-1, 1, (k, n)).astype(np.float32)).cuda()  # column-major n x k
C = torch.zeros(n, n, device="cuda")
TB.ssyrk(A, C, n, k, n, n, 1.0, 0.0, "N", 256, TB.PLAIN)
TB.synchronize()
h.update(C.cpu().numpy().tobytes())
for side, m, nn in (("L", 4096, 1536), ("R", 1536, 4096)):
    nt = m if side == "L" else nn
    L = (np.tril(g.uniform(-1, 1, (nt, nt)) / np.sqrt(nt), -1) + np.diag(g.uniform(1, 2, nt))).astype(np.float32)
    B = g.uniform(-1, 1, (m, nn)).astype(np.float32)
    for prec in (TB.PLAIN, TB.SPLIT):
        dA = torch.from_numpy(np.ascontiguousarray(L.T)).cuda()
        dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
        TB.strsm(side, dA, dB, m, nn, nt, m, 512, prec)
        TB.synchronize()
        h.update(dB.cpu().numpy().tobytes())
m = 2048
S = torch.from_numpy(g.uniform(-1, 1, (m, m)).astype(np.float32)).cuda()
Bs = torch.from_numpy(g.uniform(-1, 1, (m, m)).astype(np.float32)).cuda()
Cs = torch.from_numpy(g.uniform(-1, 1, (m, m)).astype(np.float32)).cuda()
TB._bind_stream(S)
TB._check(TB.lib.tb_ssymm(b"L", m, m, ctypes.c_float(1.0), S.data_ptr(), m, Bs.data_ptr(), m, ctypes.c_float(0.5),
                          Cs.data_ptr(), m, 0))
Cg = torch.zeros(m, m, device="cuda")
TB.sgemm("N", "T", m, m, m, 1.0, S, m, Bs, m, 0.0, Cg, m)
TB.synchronize()
h.update(Cs.cpu().numpy().tobytes())
h.update(Cg.cpu().numpy().tobytes())
print(h.hexdigest())
"""


def _digest(pdl):
    env = dict(os.environ, TB_PDL=pdl)
    out = subprocess.run([sys.executable, "-c", SCRIPT, os.path.join(ROOT, "tensor-blas_b200", "python")], env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return out.stdout.strip().splitlines()[-1]


def test_dependent_launches_are_bit_identical():
    assert _digest("1") == _digest("0")
