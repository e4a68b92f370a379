"""SYR2K, TRMM and SYMM on the GPU vs the oracle's FP64 arithmetic models
(tb_oracle.syr2k_model / trmm_model / symm_model). Inputs include the
wide-exponent distribution of the SYR2K/TRMM/SYMM configuration,
N(0,1) * 2^U(-8,8). Tolerances as in test_gpu_gemm_syrk.py."""
import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _wide(g, shape):
    return (g.standard_normal(shape) * np.exp2(g.uniform(-8, 8, shape))).astype(np.float32)


def _tol(k, precision):
    return 2e-6 if precision else 1e-6 + 1e-8 * k


def _rel(got, model, mask=None):
    _, nrm = orc.rel_errors(got, model, mask)
    return nrm


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n,k,beta,wide", [(512, 256, 0.0, False), (300, 130, 0.5, False), (640, 512, 0.0, True)])
def test_ssyr2k(tblas, n, k, beta, wide, precision):
    g = _rng(n + k)
    A = _wide(g, (n, k)) if wide else g.uniform(-1, 1, (n, k)).astype(np.float32)
    B = _wide(g, (n, k)) if wide else g.uniform(-1, 1, (n, k)).astype(np.float32)
    C0 = g.uniform(-1, 1, (n, n)).astype(np.float32)
    got = tblas.syr2k(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), 1.0, beta,
                      torch.from_numpy(C0).cuda(), precision=precision)
    tblas.synchronize()
    got = got.cpu().numpy()
    model = orc.syr2k_model(A, B, 1.0, beta, C0, split=bool(precision))
    low = np.tril(np.ones((n, n), dtype=bool))
    err = _rel(got, model, low)
    print(f"syr2k n={n} k={k} prec={precision}: {err:.3e}")
    assert err <= _tol(2 * k, precision)
    assert np.array_equal(got[~low], C0[~low])


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("uplo", ["L", "U"])
# (1100, 600): CTA-pair tiles with host-balanced ranges and a ragged last 256-band
@pytest.mark.parametrize("m,n,wide", [(512, 384, False), (333, 200, False), (768, 256, True), (1100, 600, False)])
def test_strmm(tblas, uplo, m, n, wide, precision):
    g = _rng(3 * m + n)
    A = _wide(g, (m, m)) if wide else g.uniform(-1, 1, (m, m)).astype(np.float32)
    A_garbage = A.copy()
    if uplo == "L":
        A_garbage[np.triu_indices(m, 1)] = np.nan  # never read
    else:
        A_garbage[np.tril_indices(m, -1)] = np.nan
    B = _wide(g, (m, n)) if wide else g.uniform(-1, 1, (m, n)).astype(np.float32)
    got = tblas.trmm(torch.from_numpy(A_garbage).cuda(), torch.from_numpy(B).cuda(), 0.75, uplo,
                     precision=precision)
    tblas.synchronize()
    model = orc.trmm_model(A, B, 0.75, upper=(uplo == "U"), split=bool(precision))
    err = _rel(got.cpu().numpy(), model)
    print(f"trmm {uplo} m={m} n={n} prec={precision}: {err:.3e}")
    assert err <= _tol(m, precision)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("m,n,beta,wide", [(512, 256, 0.0, False), (270, 130, -1.0, False), (640, 384, 0.0, True)])
def test_ssymm(tblas, uplo, m, n, beta, wide, precision):
    g = _rng(7 * m + n)
    A = _wide(g, (m, m)) if wide else g.uniform(-1, 1, (m, m)).astype(np.float32)
    A_in = A.copy()
    if uplo == "L":
        A_in[np.triu_indices(m, 1)] = np.nan  # other triangle never read
    else:
        A_in[np.tril_indices(m, -1)] = np.nan
    B = _wide(g, (m, n)) if wide else g.uniform(-1, 1, (m, n)).astype(np.float32)
    C0 = g.uniform(-1, 1, (m, n)).astype(np.float32)
    dA = torch.from_numpy(A_in).cuda()
    got = tblas.symm(dA, torch.from_numpy(B).cuda(), 1.25, beta, torch.from_numpy(C0).cuda(), uplo,
                     precision=precision)
    tblas.synchronize()
    model = orc.symm_model(A, B, 1.25, beta, C0, lower=(uplo == "L"), split=bool(precision))
    err = _rel(got.cpu().numpy(), model)
    print(f"symm {uplo} m={m} n={n} prec={precision}: {err:.3e}")
    assert err <= _tol(m, precision)
    # A is not modified (the reference mirrors it in place)
    assert np.array_equal(dA.cpu().numpy(), A_in, equal_nan=True)
