"""Host-memory SYRK / TRSM (tb_ssyrk_host, tb_strsm_host): the panel-streamed
results must equal the device-pointer routines bit for bit (same tiles, same
K order per element), leave the strict upper triangle of C untouched, and
honour beta, ragged panel edges and both TRSM sides."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _pinned(x):
    return torch.from_numpy(np.ascontiguousarray(x)).pin_memory()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n,k,beta", [(2500, 700, 0.0), (1024, 64, 0.5), (300, 1000, 0.0), (3100, 300, -1.0)])
def test_ssyrk_host_matches_device(tblas, n, k, beta, precision):
    g = np.random.Generator(np.random.PCG64(n + k))
    A = g.uniform(-1, 1, (k, n)).astype(np.float32)      # column-major n x k
    C0 = g.uniform(-1, 1, (n, n)).astype(np.float32)     # column-major n x n
    hA, hC = _pinned(A), _pinned(C0)
    tblas.ssyrk_host(hA, hC, n, k, n, n, 1.25, beta, 256, precision)
    dA, dC = torch.from_numpy(A).cuda(), torch.from_numpy(C0).cuda()
    tblas.ssyrk(dA, dC, n, k, n, n, 1.25, beta, "N", 256, precision)
    tblas.synchronize()
    got, ref = hC.numpy(), dC.cpu().numpy()
    # storage [j, i] holds C(i, j): the lower triangle is the storage's upper
    up = np.triu(np.ones((n, n), dtype=bool))
    assert np.array_equal(got[up], ref[up])
    assert np.array_equal(got[~up], C0[~up])  # strict upper of C untouched


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("side,m,n,nb", [("L", 3000, 2100, 512), ("R", 2100, 3000, 512), ("L", 700, 1500, 256),
                                         ("R", 1500, 700, 128), ("L", 4096, 64, 512)])
def test_strsm_host_matches_device(tblas, side, m, n, nb, precision):
    g = np.random.Generator(np.random.PCG64(m * 7 + n))
    nt = n if side == "R" else m
    L = np.tril(g.uniform(-1, 1, (nt, nt)) / np.sqrt(nt), -1) + np.diag(g.uniform(1, 2, nt))
    A = np.ascontiguousarray(L.T).astype(np.float32)     # column-major lower A
    A[np.tril(np.ones((nt, nt), dtype=bool), -1)] = np.nan  # storage lower = A's strict upper: never read
    B = g.uniform(-1, 1, (n, m)).astype(np.float32)      # column-major m x n
    hA, hB = _pinned(A), _pinned(B)
    tblas.strsm_host(side, hA, hB, m, n, nt, m, nb, precision)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    tblas.strsm(side, dA, dB, m, n, nt, m, nb, precision)
    tblas.synchronize()
    got, ref = hB.numpy(), dB.cpu().numpy()
    assert np.all(np.isfinite(got))
    assert np.array_equal(got, ref)


def test_host_api_rejects_device_tensors(tblas):
    d = torch.zeros(4, 4, device="cuda")
    with pytest.raises(TypeError):
        tblas.ssyrk_host(d, d, 4, 4, 4, 4)


HOST_CONVERT = r"""
import hashlib, sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
import TensorBLAS as TB
n, k, beta = int(sys.argv[2]), int(sys.argv[3]), float(sys.argv[4])
g = np.random.Generator(np.random.PCG64(n + k))
A = g.uniform(-1, 1, (k, n)).astype(np.float32)
C0 = g.uniform(-1, 1, (n, n)).astype(np.float32)
hA, hC = torch.from_numpy(A).pin_memory(), torch.from_numpy(C0).pin_memory()
TB.ssyrk_host(hA, hC, n, k, n, n, 1.25, beta, 256, TB.PLAIN)
dA, dC = torch.from_numpy(A).cuda(), torch.from_numpy(C0).cuda()
TB.ssyrk(dA, dC, n, k, n, n, 1.25, beta, "N", 256, TB.PLAIN)
TB.synchronize()
print(int(np.array_equal(hC.numpy(), dC.cpu().numpy())))
"""


@pytest.mark.parametrize("every", ["1", "2"])
@pytest.mark.parametrize("n,k,beta", [(3100, 700, 0.0), (2048, 1000, 0.5)])
def test_ssyrk_host_with_host_side_conversion(every, n, k, beta):
    """TB_HOST_F16_EVERY converts every (or every second) A panel to FP16 on
    the host's cores before it crosses PCIe: the result must still equal the
    device routine's bit for bit (read once per process: a subprocess)."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, TB_HOST_F16_EVERY=every)
    r = subprocess.run([sys.executable, "-c", HOST_CONVERT, os.path.join(root, "tensor-blas_b200", "python"), str(n),
                        str(k), str(beta)], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "1"
