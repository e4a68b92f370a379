"""GEMM engine and SYRK on the GPU vs the oracle's FP64 arithmetic model.

Tolerances: the oracle evaluates the same FP16-rounded (plain) or hi/lo split
(split) products exactly in FP64, so what remains is the FP32 accumulation.
Plain mode accumulates a tile's whole K inside the tensor core, whose FP32
adds truncate: error grows ~ (K/16) * 2^-24, hence normwise
<= 1e-6 + 1e-8 * K.  Split mode folds every 128 K into round-to-nearest FP32
registers: normwise <= 2e-6.  Per element,
|C - C_model| <= e(K) * sum_p |a_ip b_jp| + tiny, with e = 2e-6 + 2e-8 * K
(plain) and 1e-5 (split).
"""
import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu

def elem_tol(k, precision):
    return 1e-5 if precision else 2e-6 + 2e-8 * k


def norm_tol(k, precision):
    return 2e-6 if precision else 1e-6 + 1e-8 * k


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _check(got, model, absprod, tol, etol, mask=None):
    got = np.asarray(got, dtype=np.float64)
    if mask is None:
        mask = np.ones(got.shape, dtype=bool)
    d = np.abs(got - model)[mask]
    bound = etol * absprod[mask] + 1e-30
    worst = float(np.max(d / bound)) if d.size else 0.0
    _, nrm = orc.rel_errors(got, model, mask)
    print(f"normwise {nrm:.3e} (tol {tol:.1e}) elementwise ratio {worst:.3f}")
    assert nrm <= tol, f"normwise {nrm:.3e}"
    assert worst <= 1.0, f"elementwise bound exceeded x{worst:.2f}"
    return nrm


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("m,n,k,ldc_pad", [(256, 512, 128, 0), (1000, 300, 200, 0), (129, 257, 65, 0),
                                           (256, 300, 128, 1), (384, 256, 1024, 4)])
def test_sgemm(tblas, ta, tb, m, n, k, ldc_pad, precision):
    """ldc_pad = 1 makes C unreachable for TMA (per-element epilogue path)."""
    rng = _rng(1000 + m + n + k)
    opA = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    opB = rng.uniform(-1, 1, (k, n)).astype(np.float32)
    C0 = rng.uniform(-1, 1, (m, n)).astype(np.float32)
    alpha, beta = 1.5, -0.5
    A_st = opA if ta == "N" else opA.T.copy()   # stored (column-major) matrix
    B_st = opB if tb == "N" else opB.T.copy()
    dA = torch.from_numpy(np.ascontiguousarray(A_st.T)).cuda()  # row-major storage of A_st^T == col-major A_st
    dB = torch.from_numpy(np.ascontiguousarray(B_st.T)).cuda()
    ldc = m + ldc_pad
    Cpad = np.full((n, ldc), 7.0, dtype=np.float32)
    Cpad[:, :m] = C0.T
    dC = torch.from_numpy(Cpad).cuda()
    lda, ldb = A_st.shape[0], B_st.shape[0]
    tblas._check(tblas.lib.tb_sgemm(ta.encode(), tb.encode(), m, n, k, alpha, dA.data_ptr(), lda, dB.data_ptr(),
                                    ldb, beta, dC.data_ptr(), ldc, precision))
    tblas.synchronize()
    full = dC.cpu().numpy()
    assert np.all(full[:, m:] == 7.0), "padding rows of C were written"
    got = full[:, :m].T
    if precision == 0:
        prod = orc.h(opA) @ orc.h(opB)
    else:
        prod = orc.split_product(opA, opB)
    model = alpha * prod + beta * C0.astype(np.float64)
    absprod = abs(alpha) * (np.abs(opA.astype(np.float64)) @ np.abs(opB.astype(np.float64))) + abs(beta) * np.abs(C0)
    _check(got, model, absprod, norm_tol(k, precision), elem_tol(k, precision))


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("n,k,beta", [(4096, 4096, 0.0), (1000, 300, 0.75), (130, 70, 0.0), (1, 5, 0.0)])
def test_ssyrk(tblas, trans, n, k, beta, precision):
    rng = _rng(7 + n + k)
    A = rng.uniform(-1, 1, (n, k)).astype(np.float32)      # logical op(A), n x k
    C0 = rng.uniform(-1, 1, (n, n)).astype(np.float32)
    alpha = 1.0
    A_st = A if trans == "N" else A.T.copy()
    dA = torch.from_numpy(np.ascontiguousarray(A_st.T)).cuda()
    dC = torch.from_numpy(np.ascontiguousarray(C0.T)).cuda()
    lda = A_st.shape[0]
    tblas._check(tblas.lib.tb_ssyrk(b"L", trans.encode(), n, k, alpha, dA.data_ptr(), lda, beta, dC.data_ptr(), n,
                                    256, precision))
    tblas.synchronize()
    got = dC.cpu().numpy().T
    model = orc.syrk_model(A, alpha, beta, C0, split=bool(precision))
    A64 = np.abs(A.astype(np.float64))
    absprod = A64 @ A64.T + abs(beta) * np.abs(C0)
    low = np.tril(np.ones((n, n), dtype=bool))
    _check(got, model, absprod, norm_tol(k, precision), elem_tol(k, precision), low)
    # strict upper triangle untouched
    assert np.array_equal(got[~low], C0[~low])


def test_tc_syrk_python_api(tblas):
    """The reference's python entry: C = A A^T, full symmetric (python/TensorBLAS.py:11-34)."""
    rng = _rng(3)
    A = torch.from_numpy(rng.uniform(-1, 1, (777, 513)).astype(np.float32)).cuda()
    C = tblas.tc_syrk(A, nb=256)
    torch.cuda.synchronize()
    An = A.cpu().numpy()
    model = orc.h(An) @ orc.h(An).T
    got = C.cpu().numpy()
    assert np.array_equal(got, got.T)
    _, nrm = orc.rel_errors(got, model)
    assert nrm <= norm_tol(513, 0)
    Ct = tblas.tc_syrk(A, transpose=True, nb=256)
    torch.cuda.synchronize()
    model_t = orc.h(An).T @ orc.h(An)
    _, nrm = orc.rel_errors(Ct.cpu().numpy(), model_t)
    assert nrm <= norm_tol(777, 0)
