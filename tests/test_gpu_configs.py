"""Parity at the full sizes of the benchmark configurations.

Each case runs the routine on seeded synthetic inputs of the configuration's
shape and value distribution and checks sampled entries against an FP64 (or,
for the FP64 routines, long double) evaluation on the host, with the bound
written in the test:

  * SYRK n = k = 16384 (nb 256) and TRSM m = n = 16384 (nb 512, left and
    right side; A off-diagonal U[-1,1]/sqrt(n), diagonal U[1,2]), plain and
    split, plus agreement of the plain outputs with the reference library's
    own tc_syrk / tc_trsm on the same inputs when its build (oracle/_ref) is
    present;
  * SYR2K n = 16384, k = 4096, TRMM (left, upper) and SYMM (left, lower)
    m = n = 16384 on entries N(0,1) 2^U(-8,8): plain, split and FP8;
  * FP64 DSYRK n = k = 8192 on the INT8 Ozaki engine, A = N(0,1)
    exp(phi N(0,1)) for phi in {0.5, 2}, with the slice count the library
    picks itself;
  * 512 independent SYRK / TRSM instances of order log-uniform in
    [64, 2048] as one grouped batch, plain and split, every instance checked.
"""
import ctypes
import os

import numpy as np
import pytest
import torch
from scipy.linalg import solve_triangular

import tb_oracle as orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libTensorBLAS_ref.so")
N = 16384
P, L, F = ctypes.c_void_p, ctypes.c_long, ctypes.c_float

# normwise relative error bounds vs FP64 (sampled)
BOUND = {"plain": 1e-3, "split": 1e-6, "fp8": 6e-2}


def _ref_lib():
    if not os.path.exists(REF_SO):
        return None
    lib = ctypes.CDLL(REF_SO)
    lib.ref_syrk.argtypes = [L, L, F, P, F, P, L]
    lib.ref_trsm.argtypes = [L, L, P, P, L]
    return lib


def _norm_rel(got, ref):
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))


def _tri_inputs(n, seed):
    """Column-major lower-triangular A (torch storage = A^T) as in the TRSM configuration."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    Lw = torch.rand(n, n, device="cuda", generator=g) * 2 - 1
    Lw = torch.tril(Lw, -1) / n ** 0.5 + torch.diag(torch.rand(n, device="cuda", generator=g) + 1)
    T = Lw.t().contiguous()
    del Lw
    B = torch.rand(n, n, device="cuda", generator=g) * 2 - 1
    return T, B


@pytest.fixture(scope="module")
def trsm_inputs():
    T, B0 = _tri_inputs(N, 2718)
    Lh = T.cpu().numpy().T.astype(np.float64)   # logical lower-triangular A
    Bh = B0.cpu().numpy().T.astype(np.float64)  # logical B
    yield T, B0, Lh, Bh
    del T, B0
    torch.cuda.empty_cache()


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("prec", ["plain", "split"])
def test_trsm_16384_nb512_vs_fp64(tblas, trsm_inputs, side, prec):
    T, B0, Lh, Bh = trsm_inputs
    X = B0.clone()
    tblas._bind_stream(X)
    tblas._check(tblas.lib.tb_strsm(side.encode(), N, N, T.data_ptr(), N, X.data_ptr(), N, 512,
                                    tblas.PLAIN if prec == "plain" else tblas.SPLIT))
    tblas.synchronize()
    Xh = X.cpu().numpy().T.astype(np.float64)
    g = np.random.Generator(np.random.PCG64(11))
    idx = g.integers(0, N, 32)
    if side == "L":   # A x_j = b_j for 32 columns
        ref = solve_triangular(Lh, Bh[:, idx], lower=True)
        got = Xh[:, idx]
    else:             # x_i A^T = b_i  <=>  A x_i^T = b_i^T for 32 rows
        ref = solve_triangular(Lh, Bh[idx, :].T, lower=True)
        got = Xh[idx, :].T
    err = _norm_rel(got, ref)
    print(f"TRSM 16384 side {side} {prec}: normwise {err:.3e} (32 sampled {'columns' if side == 'L' else 'rows'})")
    assert err <= BOUND[prec]


def test_trsm_16384_agrees_with_reference_tc_trsm(tblas, trsm_inputs):
    ref = _ref_lib()
    if ref is None:
        pytest.skip("reference build oracle/_ref not present")
    T, B0, Lh, Bh = trsm_inputs
    X = B0.clone()
    tblas._bind_stream(X)
    tblas._check(tblas.lib.tb_strsm(b"R", N, N, T.data_ptr(), N, X.data_ptr(), N, 512, tblas.PLAIN))
    tblas.synchronize()
    hT = np.ascontiguousarray(T.cpu().numpy())
    hX = np.ascontiguousarray(B0.cpu().numpy())
    assert ref.ref_trsm(N, N, hT.ctypes.data_as(P), hX.ctypes.data_as(P), 512) == 0
    mine = X.cpu().numpy().astype(np.float64)
    theirs = hX.astype(np.float64)
    agree = _norm_rel(mine, theirs)
    g = np.random.Generator(np.random.PCG64(12))
    idx = g.integers(0, N, 16)
    exact = solve_triangular(Lh, Bh[idx, :].T, lower=True).T   # rows of X (storage is X^T)
    e_mine = _norm_rel(mine.T[idx, :], exact)
    e_ref = _norm_rel(theirs.T[idx, :], exact)
    print(f"TRSM 16384 plain vs reference tc_trsm: normwise {agree:.3e}; vs FP64 mine {e_mine:.3e} "
          f"reference {e_ref:.3e}")
    assert agree <= 2 * (e_mine + e_ref) + 1e-6
    assert e_mine <= 2 * e_ref


@pytest.fixture(scope="module")
def syrk_inputs():
    g = torch.Generator(device="cuda")
    g.manual_seed(1234)
    A = torch.rand(N, N, device="cuda", generator=g) * 2 - 1   # column-major n x k storage
    yield A
    del A
    torch.cuda.empty_cache()


def _syrk_sample(A, C, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    Ah = A.cpu().numpy().astype(np.float64)   # Ah[p, i] = A(i, p)
    i, j = g.integers(0, N, 4096), g.integers(0, N, 4096)
    lo, hi = np.maximum(i, j), np.minimum(i, j)
    ref = np.einsum("pk,pk->k", Ah[:, lo], Ah[:, hi])
    got = C.cpu().numpy()[hi, lo].astype(np.float64)
    return got, ref


@pytest.mark.parametrize("prec", ["plain", "split"])
def test_syrk_16384_vs_fp64(tblas, syrk_inputs, prec):
    A = syrk_inputs
    C = torch.zeros(N, N, device="cuda")
    tblas._bind_stream(A)
    tblas._check(tblas.lib.tb_ssyrk(b"L", b"N", N, N, 1.0, A.data_ptr(), N, 0.0, C.data_ptr(), N, 256,
                                    tblas.PLAIN if prec == "plain" else tblas.SPLIT))
    tblas.synchronize()
    got, ref = _syrk_sample(A, C, 3)
    err = _norm_rel(got, ref)
    print(f"SYRK 16384 {prec}: normwise {err:.3e} (4096 sampled lower entries)")
    assert err <= BOUND[prec]
    assert torch.count_nonzero(torch.triu(C.t(), 1)) == 0  # the strict upper triangle is never written


def test_syrk_16384_agrees_with_reference_tc_syrk(tblas, syrk_inputs):
    ref = _ref_lib()
    if ref is None:
        pytest.skip("reference build oracle/_ref not present")
    A = syrk_inputs
    C = torch.zeros(N, N, device="cuda")
    tblas._bind_stream(A)
    tblas._check(tblas.lib.tb_ssyrk(b"L", b"N", N, N, 1.0, A.data_ptr(), N, 0.0, C.data_ptr(), N, 256, tblas.PLAIN))
    tblas.synchronize()
    hA = np.ascontiguousarray(A.cpu().numpy())
    hC = np.zeros((N, N), dtype=np.float32)
    assert ref.ref_syrk(N, N, 1.0, hA.ctypes.data_as(P), 0.0, hC.ctypes.data_as(P), 256) == 0
    mine = torch.tril(C.t()).cpu().numpy().astype(np.float64)     # logical lower triangle
    theirs = np.tril(hC.T).astype(np.float64)
    agree = _norm_rel(mine, theirs)
    got, exact = _syrk_sample(A, C, 4)
    e_mine = _norm_rel(got, exact)
    g = np.random.Generator(np.random.PCG64(4))
    i, j = g.integers(0, N, 4096), g.integers(0, N, 4096)
    lo, hi = np.maximum(i, j), np.minimum(i, j)
    e_ref = _norm_rel(hC[hi, lo].astype(np.float64), exact)
    print(f"SYRK 16384 plain vs reference tc_syrk: normwise {agree:.3e}; vs FP64 mine {e_mine:.3e} "
          f"reference {e_ref:.3e}")
    # both round the same FP16 operands: they differ only in the order and
    # truncation of the FP32 accumulation (each within 1e-6 + 1e-8 K of the
    # exact product of the rounded operands)
    assert agree <= 2 * (1e-6 + 1e-8 * N)
    assert e_mine <= 2 * e_ref


def _wide(g, r, c):
    x = torch.randn(r, c, device="cuda", generator=g)
    return x * torch.exp2(torch.rand(r, c, device="cuda", generator=g) * 16 - 8)


PRECS = [("plain", 0), ("split", 1), ("fp8", 2)]


def test_syr2k_16384x4096_vs_fp64(tblas):
    g = torch.Generator(device="cuda")
    g.manual_seed(99)
    n, k = N, 4096
    A, B = _wide(g, k, n), _wide(g, k, n)   # column-major n x k
    C = torch.zeros(n, n, device="cuda")
    Ah, Bh = A.cpu().numpy().astype(np.float64), B.cpu().numpy().astype(np.float64)
    rng = np.random.Generator(np.random.PCG64(5))
    i, j = rng.integers(0, n, 512), rng.integers(0, n, 512)
    lo, hi = np.maximum(i, j), np.minimum(i, j)
    ref = np.einsum("pk,pk->k", Ah[:, lo], Bh[:, hi]) + np.einsum("pk,pk->k", Bh[:, lo], Ah[:, hi])
    tblas._bind_stream(A)
    for name, prec in PRECS:
        tblas._check(tblas.lib.tb_ssyr2k(b"L", b"N", n, k, 1.0, A.data_ptr(), n, B.data_ptr(), n, 0.0, C.data_ptr(), n,
                                         256, prec))
        tblas.synchronize()
        err = _norm_rel(C.cpu().numpy()[hi, lo].astype(np.float64), ref)
        print(f"SYR2K 16384x4096 {name}: normwise {err:.3e}")
        assert err <= BOUND[name], name


def test_trmm_upper_and_symm_16384_vs_fp64(tblas):
    g = torch.Generator(device="cuda")
    g.manual_seed(98)
    m = n = N
    A, B = _wide(g, m, m), _wide(g, n, m)   # A m x m, B m x n (column-major)
    C = torch.zeros(n, m, device="cuda")
    An, Bn = A.cpu().numpy(), B.cpu().numpy()   # An[p, i] = A(i, p); Bn[j, p] = B(p, j)
    rng = np.random.Generator(np.random.PCG64(6))
    i, j = rng.integers(0, m, 128), rng.integers(0, n, 128)
    ref_trmm = np.array([np.dot(An[ii:, ii].astype(np.float64), Bn[jj, ii:].astype(np.float64))
                         for ii, jj in zip(i, j)])
    ref_symm = np.array([np.dot(np.concatenate([An[:ii + 1, ii], An[ii, ii + 1:]]).astype(np.float64),
                                Bn[jj, :].astype(np.float64)) for ii, jj in zip(i, j)])
    tblas._bind_stream(A)
    for name, prec in PRECS:
        tblas._check(tblas.lib.tb_strmm(b"U", m, n, 1.0, A.data_ptr(), m, B.data_ptr(), m, C.data_ptr(), m, 256, prec))
        tblas.synchronize()
        e1 = _norm_rel(C.cpu().numpy()[j, i].astype(np.float64), ref_trmm)
        tblas._check(tblas.lib.tb_ssymm(b"L", m, n, 1.0, A.data_ptr(), m, B.data_ptr(), m, 0.0, C.data_ptr(), m, prec))
        tblas.synchronize()
        e2 = _norm_rel(C.cpu().numpy()[j, i].astype(np.float64), ref_symm)
        print(f"TRMM upper 16384 {name}: normwise {e1:.3e}; SYMM lower 16384 {name}: normwise {e2:.3e}")
        assert e1 <= BOUND[name] and e2 <= BOUND[name], name


@pytest.mark.parametrize("phi", [0.5, 2.0])
def test_dsyrk_ozaki_8192_auto_slices_vs_long_double(tblas, phi):
    n = k = 8192
    g = np.random.Generator(np.random.PCG64(17))
    Ah = g.standard_normal((n, k)) * np.exp(phi * g.standard_normal((n, k)))
    dA = torch.from_numpy(np.ascontiguousarray(Ah.T)).cuda()
    dC = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    lib = tblas.lib
    lib.tb_dsyrk_ozaki.argtypes = [ctypes.c_char, ctypes.c_char, L, L, ctypes.c_double, P, L, ctypes.c_double, P, L,
                                   ctypes.c_int]
    tblas._bind_stream(dA)
    tblas._check(lib.tb_dsyrk_ozaki(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, 0))
    tblas.synchronize()
    Ch = dC.cpu().numpy().T
    r, c = g.integers(0, n, 2000), g.integers(0, n, 2000)
    lo, hi = np.maximum(r, c), np.minimum(r, c)
    ex = orc.syrk_extended(Ah, lo, hi)
    d = np.abs(Ch[lo, hi] - ex).astype(np.float64)
    err = float(np.linalg.norm(d) / np.linalg.norm(ex.astype(np.float64)))
    print(f"DSYRK 8192 Ozaki phi={phi} (automatic slices): normwise {err:.3e} vs long double")
    assert err <= 1e-14


@pytest.mark.parametrize("prec", ["plain", "split"])
def test_batch_512_uneven_vs_fp64(tblas, prec):
    g = np.random.Generator(np.random.PCG64(2025))
    ns = np.round(np.exp(g.uniform(np.log(64), np.log(2048), 512))).astype(int)
    tg = torch.Generator(device="cuda")
    tg.manual_seed(77)
    kinds, As, BC, B0 = [], [], [], []
    for i, m in enumerate(ns):
        if i % 2 == 0:
            a = torch.rand(m, m, device="cuda", generator=tg) * 2 - 1
            bc = torch.zeros(m, m, device="cuda")
        else:
            lt = torch.tril(torch.rand(m, m, device="cuda", generator=tg) * 2 - 1, -1) / m ** 0.5
            a = (lt + torch.diag(torch.rand(m, device="cuda", generator=tg) + 1)).t().contiguous()
            bc = torch.rand(m, m, device="cuda", generator=tg) * 2 - 1
        kinds.append(i % 2)
        As.append(a)
        BC.append(bc)
        B0.append(bc.cpu().numpy().T.astype(np.float64))
    batch = tblas.Batch(kinds, As, BC, precision=tblas.PLAIN if prec == "plain" else tblas.SPLIT)
    try:
        batch.run()
        tblas.synchronize()
    finally:
        batch.close()
    worst = {0: 0.0, 1: 0.0}
    for kind, a, bc, b0, m in zip(kinds, As, BC, B0, ns):
        A = a.cpu().numpy().T.astype(np.float64)   # logical matrix
        got = bc.cpu().numpy().T.astype(np.float64)
        if kind == 0:
            ref = A @ A.T
            low = np.tril(np.ones((m, m), dtype=bool))
            e = float(np.linalg.norm((got - ref)[low]) / np.linalg.norm(ref[low]))
        else:   # X A^T = B
            ref = solve_triangular(A, b0.T, lower=True).T
            e = _norm_rel(got, ref)
        worst[kind] = max(worst[kind], e)
    print(f"batch 512 {prec}: worst normwise SYRK {worst[0]:.3e}, TRSM {worst[1]:.3e}")
    assert worst[0] <= BOUND[prec] and worst[1] <= BOUND[prec]
