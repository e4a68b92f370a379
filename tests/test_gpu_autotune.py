"""nb = TB_NB_AUTO on the GPU: the first call tunes (one cache entry per
key, nb from the candidate set), later calls reuse the entry, and the
results are those of the routine run with explicit parameters (checked
against the oracle model / the FP64 solution like the routine tests)."""
import numpy as np
import pytest
import torch

import tb_oracle as orc
import TensorBLAS as TB

pytestmark = pytest.mark.gpu


@pytest.fixture()
def fresh():
    TB.autotune_set_file(None)
    TB.lib.tb_autotune_clear()
    yield
    TB.lib.tb_autotune_clear()


def test_ssyrk_auto(fresh):
    g = np.random.Generator(np.random.PCG64(41))
    n, k = 1024, 768
    A = g.uniform(-1, 1, (n, k)).astype(np.float32)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()  # column-major n x k
    for rep in range(2):
        dC = torch.zeros(n * n, device="cuda")
        TB.ssyrk(dA, dC, n, k, n, n, 1.0, 0.0, "N", TB.NB_AUTO, TB.SPLIT)
        TB.synchronize()
        assert TB.autotune_entries() == 1
    choice = TB.autotune_get("ssyrk", "LN", n, k, TB.SPLIT)
    assert choice is not None and choice[1] in (0, 1)
    got = dC.cpu().numpy().reshape(n, n).T.astype(np.float64)
    exact = A.astype(np.float64) @ A.astype(np.float64).T
    low = np.tril(np.ones((n, n), dtype=bool))
    err = np.linalg.norm((got - exact)[low]) / np.linalg.norm(exact[low])
    assert err <= 2e-6


def test_strsm_auto(fresh):
    g = np.random.Generator(np.random.PCG64(43))
    m, n = 2048, 512
    A = (np.tril(g.uniform(-1, 1, (m, m)) / np.sqrt(m), -1) + np.diag(g.uniform(1, 2, m))).astype(np.float32)
    B = g.uniform(-1, 1, (m, n)).astype(np.float32)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    TB.strsm("L", dA, dB, m, n, m, m, TB.NB_AUTO, TB.SPLIT)
    TB.synchronize()
    nb, engine = TB.autotune_get("strsm", "L", m, n, TB.SPLIT)
    assert nb in (128, 256, 512) and engine in (0, 1)
    X = dB.cpu().numpy().T.astype(np.float64)
    exact = np.linalg.solve(A.astype(np.float64), B.astype(np.float64))
    _, err = orc.rel_errors(X, exact)
    assert err <= 2e-6
    # the same call again reuses the entry and gives the same result as the
    # explicit (nb, engine) it chose
    dB2 = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    TB.strsm("L", dA, dB2, m, n, m, m, TB.NB_AUTO, TB.SPLIT)
    TB.synchronize()
    assert TB.autotune_entries() == 1
    assert torch.equal(dB, dB2)
