"""Ozaki-INT8 FP64 SYRK on the GPU: slicing and INT32 slice-pair products
bit-exact against the oracle's integer arithmetic; the FP64 result against
long-double (64-bit mantissa) sums of A A^T."""
import ctypes

import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu


def _A(seed, n, k, phi):
    g = np.random.Generator(np.random.PCG64(seed))
    return g.standard_normal((n, k)) * np.exp(phi * g.standard_normal((n, k)))


def _lib(tblas):
    lib = tblas.lib
    P = ctypes.c_void_p
    L = ctypes.c_long
    lib.tb_ozaki_slice.argtypes = [L, L, P, L, ctypes.c_int, P, L, P]
    lib.tb_ozaki_level_product.argtypes = [L, L, P, L, ctypes.c_int, ctypes.c_int, P, L]
    lib.tb_dsyrk_ozaki.argtypes = [ctypes.c_char, ctypes.c_char, L, L, ctypes.c_double, P, L, ctypes.c_double, P, L,
                                   ctypes.c_int]
    return lib


@pytest.mark.parametrize("n,k,S,phi", [(300, 200, 8, 2.0), (129, 1000, 14, 0.5), (64, 16, 3, 0.0)])
def test_slices_bit_exact(tblas, n, k, S, phi):
    lib = _lib(tblas)
    A = _A(n + k, n, k, phi)
    A[3] = 0.0  # a zero row
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()  # column-major n x k
    ldq = ((k + 15) // 16) * 16
    dQ = torch.zeros(S * n * ldq, dtype=torch.int8, device="cuda")
    de = torch.zeros(n, dtype=torch.int32, device="cuda")
    tblas._check(lib.tb_ozaki_slice(n, k, dA.data_ptr(), n, S, dQ.data_ptr(), ldq, de.data_ptr()))
    tblas.synchronize()
    Q = dQ.cpu().numpy().reshape(S, n, ldq)[:, :, :k]
    e = de.cpu().numpy().astype(np.int64)
    Qr, er = orc.ozaki_slices(A, S)
    e = np.where(e < -1000, 0, e)
    assert np.array_equal(e, er)
    assert np.array_equal(Q, Qr)


@pytest.mark.parametrize("n,k,S", [(256, 384, 6), (300, 130, 4)])
def test_level_products_bit_exact(tblas, n, k, S):
    lib = _lib(tblas)
    A = _A(7 * n + k, n, k, 1.0)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    Q, _ = orc.ozaki_slices(A, S)
    low = np.tril(np.ones((n, n), dtype=bool))
    for L in range(2, S + 2):
        dP = torch.zeros(n * n, dtype=torch.int32, device="cuda")
        tblas._check(lib.tb_ozaki_level_product(n, k, dA.data_ptr(), n, S, L, dP.data_ptr(), n))
        tblas.synchronize()
        P = dP.cpu().numpy().reshape(n, n).T.astype(np.int64)  # column-major
        ref = orc.ozaki_level_product(Q, L)
        assert np.array_equal(P[low], ref[low]), f"level {L}"


@pytest.mark.parametrize("n,k,phi,S,tol", [(512, 1024, 0.5, 8, 1e-14), (384, 2048, 2.0, 11, 1e-14),
                                           (200, 300, 2.0, 6, 1e-9)])
def test_dsyrk_ozaki_accuracy(tblas, n, k, phi, S, tol):
    lib = _lib(tblas)
    A = _A(n * 3 + k, n, k, phi)
    C0 = np.random.default_rng(5).standard_normal((n, n))
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dC = torch.from_numpy(np.ascontiguousarray(C0.T)).cuda()
    tblas._check(lib.tb_dsyrk_ozaki(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, S))
    tblas.synchronize()
    C = dC.cpu().numpy().T
    r, c = np.tril_indices(n)
    ex = orc.syrk_extended(A, r, c)
    d = np.abs(C[r, c] - ex)
    err = float(np.linalg.norm(d.astype(np.float64)) / np.linalg.norm(ex.astype(np.float64)))
    model = orc.ozaki_syrk_model(A, S)[r, c]
    err_model = float(np.linalg.norm((C[r, c] - model).astype(np.float64)) / np.linalg.norm(ex.astype(np.float64)))
    print(f"ozaki n={n} k={k} phi={phi} S={S}: vs long double {err:.3e}, vs Ozaki model {err_model:.3e}")
    assert err <= tol
    assert err_model <= 1e-15
    assert np.array_equal(np.triu(C, 1), np.triu(C0, 1))  # strict upper untouched


def test_dsyrk_ozaki_beta(tblas):
    lib = _lib(tblas)
    n, k = 256, 256
    A = _A(11, n, k, 0.5)
    C0 = np.random.default_rng(6).standard_normal((n, n))
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dC = torch.from_numpy(np.ascontiguousarray(C0.T)).cuda()
    tblas._check(lib.tb_dsyrk_ozaki(b"L", b"N", n, k, -0.5, dA.data_ptr(), n, 2.0, dC.data_ptr(), n, 10))
    tblas.synchronize()
    C = dC.cpu().numpy().T
    ref = -0.5 * (A @ A.T) + 2.0 * C0
    low = np.tril(np.ones((n, n), dtype=bool))
    err = np.linalg.norm((C - ref)[low]) / np.linalg.norm(ref[low])
    assert err <= 1e-14
