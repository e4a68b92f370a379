"""General BLAS flags beyond the reference's own forms (which are SYRK
lower, TRMM left/lower, TRSM right/lower/transpose, all non-unit): upper
SYRK (plain, split, FP8, FP64 Ozaki) and TRMM / TRSM for every side, uplo,
transa and diag, against the oracle's FP16 models and FP64 solves."""
import ctypes

import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu
c_, L_, F_, P_, D_, I_ = ctypes.c_char, ctypes.c_long, ctypes.c_float, ctypes.c_void_p, ctypes.c_double, ctypes.c_int


def _lib(tblas):
    lib = tblas.lib
    lib.tb_ssyrk.argtypes = [c_, c_, L_, L_, F_, P_, L_, F_, P_, L_, L_, I_]
    lib.tb_dsyrk_ozaki.argtypes = [c_, c_, L_, L_, D_, P_, L_, D_, P_, L_, I_]
    lib.tb_strmm_ex.argtypes = [c_, c_, c_, c_, L_, L_, F_, P_, L_, P_, L_, P_, L_, I_]
    lib.tb_strsm_ex.argtypes = [c_, c_, c_, c_, L_, L_, P_, L_, P_, L_, L_, I_]
    return lib


def _dev(x, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype).T)).cuda()


def _host(d):
    return d.cpu().numpy().T.astype(np.float64)


def _rel(got, ref, mask=None):
    d, r = np.asarray(got, np.float64) - ref, np.asarray(ref, np.float64)
    if mask is not None:
        d, r = d[mask], r[mask]
    return float(np.linalg.norm(d) / np.linalg.norm(r))


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_syrk_upper(tblas, precision, trans):
    lib = _lib(tblas)
    n, k = 333, 270
    g = np.random.Generator(np.random.PCG64(n + k + precision))
    A = g.uniform(-1, 1, (n, k)).astype(np.float32)
    C0 = g.uniform(-1, 1, (n, n)).astype(np.float32)
    dA = _dev(A if trans == "N" else A.T)
    dC = _dev(C0)
    tblas._check(lib.tb_ssyrk(b"U", trans.encode(), n, k, 1.0, dA.data_ptr(), n if trans == "N" else k, 0.5,
                              dC.data_ptr(), n, 256, precision))
    tblas.synchronize()
    C = _host(dC)
    up = np.triu(np.ones((n, n), dtype=bool))
    if precision == 2:
        model = orc.fp8_product_model(A, A) + 0.5 * C0
        tol = 1e-5
    else:
        model = orc._prod(A, A.T, bool(precision)) + 0.5 * C0
        tol = 2e-6 if precision else 1e-6 + 1e-8 * k
    err = _rel(C, model, up)
    print(f"syrk U {trans} prec={precision}: {err:.3e}")
    assert err <= tol
    assert np.array_equal(C[~up], C0[~up].astype(np.float64))  # strict lower untouched


def test_dsyrk_ozaki_upper(tblas):
    lib = _lib(tblas)
    n, k = 300, 400
    g = np.random.Generator(np.random.PCG64(31))
    A = g.standard_normal((n, k))
    C0 = g.standard_normal((n, n))
    dA, dC = _dev(A, np.float64), _dev(C0, np.float64)
    tblas._check(lib.tb_dsyrk_ozaki(b"U", b"N", n, k, 2.0, dA.data_ptr(), n, -1.0, dC.data_ptr(), n, 10))
    tblas.synchronize()
    C = _host(dC)
    up = np.triu(np.ones((n, n), dtype=bool))
    ex = 2.0 * orc.gemm_extended(A, A) - C0.astype(np.longdouble)
    err = _rel(C, ex.astype(np.float64), up)
    print(f"dsyrk ozaki U: {err:.3e}")
    assert err <= 1e-14
    assert np.array_equal(C[~up], C0[~up])


def _tri(g, nt, upper, unit):
    A = g.uniform(-1, 1, (nt, nt)).astype(np.float32) / np.float32(np.sqrt(nt))
    A[np.diag_indices(nt)] = g.uniform(1, 2, nt)
    T = np.triu(A) if upper else np.tril(A)
    if unit:
        T[np.diag_indices(nt)] = 1.0
    Ag = A.copy()
    Ag[np.tril_indices(nt, -1) if upper else np.triu_indices(nt, 1)] = np.nan  # other triangle never read
    if unit:
        Ag[np.diag_indices(nt)] = np.nan  # a unit diagonal is never read
    return T, Ag


FLAGS = [(s, u, t, d) for s in "LR" for u in "LU" for t in "NT" for d in "NU"]


@pytest.mark.parametrize("side,uplo,trans,diag", FLAGS)
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_trmm_ex(tblas, side, uplo, trans, diag, precision):
    lib = _lib(tblas)
    m, n = 300, 257
    na = m if side == "L" else n
    g = np.random.Generator(np.random.PCG64(FLAGS.index((side, uplo, trans, diag))))
    T, Ag = _tri(g, na, uplo == "U", diag == "U")
    B = g.uniform(-1, 1, (m, n)).astype(np.float32)
    op = T.T if trans == "T" else T
    dA, dB = _dev(Ag), _dev(B)
    dC = torch.full((n, m), 5.0, device="cuda")
    tblas._check(lib.tb_strmm_ex(side.encode(), uplo.encode(), trans.encode(), diag.encode(), m, n, 0.5,
                                 dA.data_ptr(), na, dB.data_ptr(), m, dC.data_ptr(), m, precision))
    tblas.synchronize()
    C = _host(dC)
    if precision == 2:
        model = 0.5 * (orc.fp8_product_model(op, B.T) if side == "L" else orc.fp8_product_model(B, op.T))
        tol = 1e-5
    else:
        model = 0.5 * (orc._prod(op, B, bool(precision)) if side == "L" else orc._prod(B, op, bool(precision)))
        tol = 2e-6 if precision else 1e-6 + 1e-8 * na
    err = _rel(C, model)
    print(f"trmm {side}{uplo}{trans}{diag} prec={precision}: {err:.3e}")
    assert np.all(np.isfinite(C))
    assert err <= tol


@pytest.mark.parametrize("side,uplo,trans,diag", FLAGS)
def test_trsm_ex(tblas, side, uplo, trans, diag):
    lib = _lib(tblas)
    m, n, nb = 700, 520, 128
    nt = m if side == "L" else n
    g = np.random.Generator(np.random.PCG64(100 + FLAGS.index((side, uplo, trans, diag))))
    T, Ag = _tri(g, nt, uplo == "U", diag == "U")
    B = g.uniform(-1, 1, (m, n)).astype(np.float32)
    op = (T.T if trans == "T" else T).astype(np.float64)
    dA, dB = _dev(Ag), _dev(B)
    tblas._check(lib.tb_strsm_ex(side.encode(), uplo.encode(), trans.encode(), diag.encode(), m, n, dA.data_ptr(), nt,
                                 dB.data_ptr(), m, nb, 1))
    tblas.synchronize()
    X = _host(dB)
    ref = np.linalg.solve(op, B.astype(np.float64)) if side == "L" else np.linalg.solve(op.T, B.astype(np.float64).T).T
    err = _rel(X, ref)
    print(f"trsm {side}{uplo}{trans}{diag}: vs FP64 {err:.3e}")
    assert np.all(np.isfinite(X))
    assert err <= 2e-6


def test_trsm_ex_native_forms_match(tblas):
    """left/lower/N and right/lower/T through tb_strsm_ex equal tb_strsm."""
    lib = _lib(tblas)
    lib.tb_strsm.argtypes = [c_, L_, L_, P_, L_, P_, L_, L_, I_]
    g = np.random.Generator(np.random.PCG64(99))
    for side, trans in (("L", "N"), ("R", "T")):
        m, n = 2100, 300
        nt = m if side == "L" else n
        T, Ag = _tri(g, nt, False, False)
        B = g.uniform(-1, 1, (m, n)).astype(np.float32)
        dA, dB1, dB2 = _dev(Ag), _dev(B), _dev(B)
        tblas._check(lib.tb_strsm_ex(side.encode(), b"L", trans.encode(), b"N", m, n, dA.data_ptr(), nt,
                                     dB1.data_ptr(), m, 512, 0))
        tblas._check(lib.tb_strsm(side.encode(), m, n, dA.data_ptr(), nt, dB2.data_ptr(), m, 512, 0))
        tblas.synchronize()
        assert torch.equal(dB1, dB2)
