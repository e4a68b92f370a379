"""FP8-e4m3 per-128x128-block scaled SYRK / SYR2K / TRMM / SYMM / GEMM
(TB_PREC_FP8) against the oracle's block-quantisation model (same scales,
same e4m3 rounding; only the FP32 summation order differs) and, for the
record, against FP64 on wide-range inputs N(0,1) * 2^U(-8,8)."""
import ctypes

import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu
FP8 = 2


def _wide(seed, shape):
    g = np.random.Generator(np.random.PCG64(seed))
    return (g.standard_normal(shape) * np.exp2(g.uniform(-8, 8, shape))).astype(np.float32)


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x, np.float32).T)).cuda()


def _host(d):
    return d.cpu().numpy().T.astype(np.float64)


def _rel(got, ref, mask=None):
    d, r = got - ref, ref
    if mask is not None:
        d, r = d[mask], r[mask]
    return float(np.linalg.norm(d) / np.linalg.norm(r))


def _lib(tblas):
    lib = tblas.lib
    c, L, F, P = ctypes.c_char, ctypes.c_long, ctypes.c_float, ctypes.c_void_p
    lib.tb_ssyrk.argtypes = [c, c, L, L, F, P, L, F, P, L, L, ctypes.c_int]
    lib.tb_sgemm.argtypes = [c, c, L, L, L, F, P, L, P, L, F, P, L, ctypes.c_int]
    return lib


@pytest.mark.parametrize("n,k", [(300, 200), (256, 640), (129, 1)])
def test_syrk_fp8(tblas, n, k):
    A = _wide(n + k, (n, k))
    C0 = np.random.default_rng(1).standard_normal((n, n)).astype(np.float32)
    dA, dC = _dev(A), _dev(C0)
    tblas._check(_lib(tblas).tb_ssyrk(b"L", b"N", n, k, 1.5, dA.data_ptr(), n, 0.5, dC.data_ptr(), n, 256, FP8))
    tblas.synchronize()
    C = _host(dC)
    low = np.tril(np.ones((n, n), dtype=bool))
    model = 1.5 * orc.fp8_product_model(A, A) + 0.5 * C0
    exact = 1.5 * (A.astype(np.float64) @ A.T.astype(np.float64)) + 0.5 * C0
    e_m, e_x = _rel(C, model, low), _rel(C, exact, low)
    print(f"syrk fp8 n={n} k={k}: vs model {e_m:.2e}, vs FP64 {e_x:.2e}")
    assert e_m <= 1e-5
    assert np.array_equal(np.triu(C, 1), np.triu(C0, 1).astype(np.float64))


@pytest.mark.parametrize("n,k", [(384, 300), (200, 128)])
def test_syr2k_fp8(tblas, n, k):
    A, B = _wide(n, (n, k)), _wide(k, (n, k))
    dA, dB = _dev(A), _dev(B)
    dC = torch.zeros(n, n, device="cuda")
    tblas._check(tblas.lib.tb_ssyr2k(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, dB.data_ptr(), n, 0.0, dC.data_ptr(),
                                     n, 256, FP8))
    tblas.synchronize()
    C = _host(dC)
    low = np.tril(np.ones((n, n), dtype=bool))
    pad = np.zeros((n, (-k) % 128), np.float32)
    model = orc.fp8_product_model(np.hstack([A, pad, B]), np.hstack([B, pad, A]))
    exact = A.astype(np.float64) @ B.T.astype(np.float64) + B.astype(np.float64) @ A.T.astype(np.float64)
    e_m, e_x = _rel(C, model, low), _rel(C, exact, low)
    print(f"syr2k fp8 n={n} k={k}: vs model {e_m:.2e}, vs FP64 {e_x:.2e}")
    assert e_m <= 1e-5


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("m,n", [(384, 200), (300, 77)])
def test_trmm_fp8(tblas, uplo, m, n):
    A, B = _wide(m, (m, m)), _wide(n, (m, n))
    At = np.tril(A) if uplo == "L" else np.triu(A)
    Ag = A.copy()
    Ag[(np.triu(np.ones((m, m)), 1) if uplo == "L" else np.tril(np.ones((m, m)), -1)).astype(bool)] = np.nan
    dA, dB = _dev(Ag), _dev(B)
    dC = torch.full((n, m), 3.0, device="cuda")
    tblas._check(tblas.lib.tb_strmm(uplo.encode(), m, n, 2.0, dA.data_ptr(), m, dB.data_ptr(), m, dC.data_ptr(), m,
                                    256, FP8))
    tblas.synchronize()
    C = _host(dC)
    model = 2.0 * orc.fp8_product_model(At, B.T)
    exact = 2.0 * At.astype(np.float64) @ B.astype(np.float64)
    e_m, e_x = _rel(C, model), _rel(C, exact)
    print(f"trmm fp8 {uplo} m={m} n={n}: vs model {e_m:.2e}, vs FP64 {e_x:.2e}")
    assert np.all(np.isfinite(C))
    assert e_m <= 1e-5


@pytest.mark.parametrize("uplo", ["L", "U"])
def test_symm_fp8(tblas, uplo):
    m, n = 320, 150
    A, B = _wide(3, (m, m)), _wide(4, (m, n))
    S = np.tril(A) + np.tril(A, -1).T if uplo == "L" else np.triu(A) + np.triu(A, 1).T
    C0 = np.random.default_rng(2).standard_normal((m, n)).astype(np.float32)
    dA, dB, dC = _dev(A), _dev(B), _dev(C0)
    tblas._check(tblas.lib.tb_ssymm(uplo.encode(), m, n, 1.0, dA.data_ptr(), m, dB.data_ptr(), m, -1.0, dC.data_ptr(),
                                    m, FP8))
    tblas.synchronize()
    C = _host(dC)
    model = orc.fp8_product_model(S, B.T) - C0
    exact = S.astype(np.float64) @ B.astype(np.float64) - C0
    e_m, e_x = _rel(C, model), _rel(C, exact)
    print(f"symm fp8 {uplo}: vs model {e_m:.2e}, vs FP64 {e_x:.2e}")
    assert e_m <= 1e-5


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T")])
def test_gemm_fp8(tblas, ta, tb):
    m, n, k = 300, 260, 400
    opA, opB = _wide(5, (m, k)), _wide(6, (k, n))
    A = opA if ta == "N" else opA.T
    B = opB if tb == "N" else opB.T
    dA, dB = _dev(A), _dev(B)
    dC = torch.zeros(n, m, device="cuda")
    tblas._check(_lib(tblas).tb_sgemm(ta.encode(), tb.encode(), m, n, k, 1.0, dA.data_ptr(), A.shape[0], dB.data_ptr(),
                                      B.shape[0], 0.0, dC.data_ptr(), m, FP8))
    tblas.synchronize()
    C = _host(dC)
    model = orc.fp8_product_model(opA, opB.T)
    exact = opA.astype(np.float64) @ opB.astype(np.float64)
    e_m, e_x = _rel(C, model), _rel(C, exact)
    print(f"gemm fp8 {ta}{tb}: vs model {e_m:.2e}, vs FP64 {e_x:.2e}")
    assert e_m <= 1e-5
    assert e_x <= 0.1
