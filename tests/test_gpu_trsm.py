"""TRSM on the GPU vs the oracle (right side = the reference's tc_trsm
semantics X A^T = B; left side = A X = B).

The oracle's model (tb_oracle.trsm_right_model) applies FP16-rounded
operands to every off-diagonal block product and solves the nb-wide diagonal
blocks exactly; the library's plain path differs from it only by FP32
accumulation and the FP32-accurate split leaf.  Split mode is also compared
with the exact FP64 solution.
"""
import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def make_tri(rng, n):
    """Lower-triangular A: off-diagonal U[-1,1]/sqrt(n), diagonal U[1,2]."""
    A = np.tril(rng.uniform(-1, 1, (n, n)) / np.sqrt(n), -1) + np.diag(rng.uniform(1, 2, n))
    up = np.triu(np.ones((n, n), dtype=bool), 1)
    A[up] = np.nan  # never referenced
    return A.astype(np.float32)


def _run(tblas, side, A, B, nb, precision):
    m, n = B.shape
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    tblas.strsm(side, dA, dB, m, n, A.shape[0], m, nb, precision)
    tblas.synchronize()
    return dB.cpu().numpy().T.astype(np.float64)


# (1024, 4608) / (4608, 1024): the independent dimension (columns for the
# left side, rows for the right side) reaches 4096, where TB_TRSM_STREAMS > 1
# would split the solve into parts
CASES = [(512, 1024, 256), (300, 700, 128), (1024, 2048, 512), (64, 64, 512), (130, 1, 64), (2048, 1536, 512),
         (4096, 512, 512), (512, 4096, 512), (1024, 4608, 256), (4608, 1024, 256)]


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("side", ["R", "L"])
@pytest.mark.parametrize("m,n,nb", CASES)
def test_strsm(tblas, side, m, n, nb, precision):
    rng = _rng(11 + m + 3 * n + nb)
    nt = n if side == "R" else m
    A = make_tri(rng, nt)
    B = rng.uniform(-1, 1, (m, n)).astype(np.float32)
    X = _run(tblas, side, A, B, nb, precision)
    assert np.all(np.isfinite(X))
    A0 = np.nan_to_num(A, nan=0.0).astype(np.float64)
    leaf = min(((min(nb, 512) + 63) // 64) * 64, 512)
    # orders below 2048 follow the reference's FP32 path in both precisions
    accurate = bool(precision) or nt < 2048
    if side == "R":
        model = orc.trsm_right_model(A0, B, leaf, split=accurate)
        exact = np.linalg.solve(A0, B.astype(np.float64).T).T
    else:
        model = orc.trsm_left_model(A0, B, leaf, split=accurate)
        exact = np.linalg.solve(A0, B.astype(np.float64))
    _, e_model = orc.rel_errors(X, model)
    _, e_exact = orc.rel_errors(X, exact)
    print(f"side={side} m={m} n={n} prec={precision}: vs model {e_model:.3e}  vs FP64 {e_exact:.3e}")
    assert e_model <= 2e-5
    if accurate:
        assert e_exact <= 2e-6
    else:
        assert e_exact <= 2e-3


def test_tc_trsm_python_api(tblas):
    """python/TensorBLAS.py:43-84: X @ A.T = B against torch's triangular solve."""
    rng = _rng(5)
    n, m = 768, 640
    A = torch.from_numpy(np.nan_to_num(make_tri(rng, n), nan=0.0)).cuda()
    B = torch.from_numpy(rng.uniform(-1, 1, (m, n)).astype(np.float32)).cuda()
    X = tblas.tc_trsm(A, B, nb=256)
    torch.cuda.synchronize()
    ref = torch.linalg.solve_triangular(A.double().T, B.double(), upper=True, left=False)
    err = (torch.linalg.norm(X.double() - ref) / torch.linalg.norm(ref)).item()
    print(f"tc_trsm python api normwise {err:.3e}")
    assert err <= 2e-3


@pytest.mark.parametrize("side", ["R", "L"])
@pytest.mark.parametrize("m,n,nb", [(4096, 512, 512), (512, 4096, 512), (2500, 2100, 256)])
def test_strsm_refine(tblas, side, m, n, nb):
    """Precision 3: plain solve plus one refinement sweep reaches FP32-level
    accuracy where the plain solve alone does not (orders >= 2048)."""
    rng = _rng(3 + m + 7 * n)
    nt = n if side == "R" else m
    A = make_tri(rng, nt)
    B = rng.uniform(-1, 1, (m, n)).astype(np.float32)
    A0 = np.nan_to_num(A, nan=0.0).astype(np.float64)
    exact = np.linalg.solve(A0, B.astype(np.float64).T).T if side == "R" else np.linalg.solve(A0, B.astype(np.float64))
    X_plain = _run(tblas, side, A, B, nb, 0)
    X_ref = _run(tblas, side, A, B, nb, 3)
    _, e_plain = orc.rel_errors(X_plain, exact)
    _, e_ref = orc.rel_errors(X_ref, exact)
    print(f"refine side={side} m={m} n={n}: plain {e_plain:.3e} -> refined {e_ref:.3e}")
    assert e_ref <= 2e-6
    if nt >= 2048:
        assert e_ref < 0.1 * e_plain
