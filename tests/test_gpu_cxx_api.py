"""The reference's C++ entry points (include/TensorBLAS.h:139-167 of the
reference: tc_syrk, tc_trsm, tc_syr2k, tc_trmm, tc_symm and their
tc_cumpsgemm_* forms), called by their mangled names through ctypes, give the
same bits as the C ABI calls they are built on (plain precision for tc_*,
split precision for tc_cumpsgemm_*), with and without the caller's FP16
workspace. Handles are passed as NULL: the library ignores them."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

P, L, F, I = ctypes.c_void_p, ctypes.c_long, ctypes.c_float, ctypes.c_int

# mangled name -> argument types (the reference's signatures)
SIGS = {
    "_Z7tc_syrkP13cublasContextllfPflfS1_lP6__halfl": [P, L, L, F, P, L, F, P, L, P, L],
    "_Z17tc_cumpsgemm_syrkPN9cumpsgemm13handle_structEllfPflfS2_ll": [P, L, L, F, P, L, F, P, L, L],
    "_Z7tc_trsmP13cublasContextllPflS1_lP6__halfl": [P, L, L, P, L, P, L, P, L],
    "_Z17tc_cumpsgemm_trsmP13cublasContextPN9cumpsgemm13handle_structEllPflS4_ll": [P, P, L, L, P, L, P, L, L],
    "_Z8tc_syr2kP13cublasContextllfPflS1_lfS1_lP6__halfl": [P, L, L, F, P, L, P, L, F, P, L, P, L],
    "_Z18tc_cumpsgemm_syr2kPN9cumpsgemm13handle_structEllfPflS2_lfS2_ll": [P, L, L, F, P, L, P, L, F, P, L, L],
    "_Z7tc_trmmP13cublasContextllfPflS1_lS1_lP6__halfl": [P, L, L, F, P, L, P, L, P, L, P, L],
    "_Z17tc_cumpsgemm_trmmPN9cumpsgemm13handle_structEllfPflS2_lS2_ll": [P, L, L, F, P, L, P, L, P, L, L],
    "_Z7tc_symmP13cublasContextllfPflS1_ifS1_lP6__half": [P, L, L, F, P, L, P, I, F, P, L, P],
    "_Z17tc_cumpsgemm_symmPN9cumpsgemm13handle_structEllfPflS2_ifS2_l": [P, L, L, F, P, L, P, I, F, P, L],
}


def _fn(lib, name):
    f = lib[name]
    f.argtypes = SIGS[name]
    f.restype = None
    return f


def _rand(g, r, c, scale=1.0):
    """A column-major r x c FP32 device matrix (torch storage c x r)."""
    return torch.from_numpy(np.ascontiguousarray((g.uniform(-1, 1, (r, c)) * scale).astype(np.float32).T)).cuda()


@pytest.fixture()
def env(tblas):
    tblas.lib.tb_set_stream(None)  # the reference API runs on the library's stream
    return tblas, np.random.Generator(np.random.PCG64(404))


@pytest.mark.parametrize("workspace", [False, True])
def test_tc_syrk_and_cumpsgemm_syrk(env, workspace):
    tblas, g = env
    lib = tblas.lib
    n, k = (1024, 777) if workspace else (1000, 777)  # n % 64 == 0: the workspace is large enough to be used
    A = _rand(g, n, k)
    C0 = _rand(g, n, n)
    ws = torch.empty(n * k, dtype=torch.float16, device="cuda") if workspace else None
    for name, prec in (("_Z7tc_syrkP13cublasContextllfPflfS1_lP6__halfl", 0),
                       ("_Z17tc_cumpsgemm_syrkPN9cumpsgemm13handle_structEllfPflfS2_ll", 1)):
        c1, c2 = C0.clone(), C0.clone()
        if prec == 0:
            _fn(lib, name)(None, n, k, 1.5, A.data_ptr(), n, 0.5, c1.data_ptr(), n,
                           ws.data_ptr() if ws is not None else None, 256)
        else:
            _fn(lib, name)(None, n, k, 1.5, A.data_ptr(), n, 0.5, c1.data_ptr(), n, 256)
        tblas._check(lib.tb_ssyrk(b"L", b"N", n, k, 1.5, A.data_ptr(), n, 0.5, c2.data_ptr(), n, 256, prec))
        tblas.synchronize()
        assert torch.equal(c1, c2), name


def test_tc_trsm_and_cumpsgemm_trsm(env):
    tblas, g = env
    lib = tblas.lib
    m, n = 2300, 2560  # order >= 2048: the plain path really is FP16
    T = np.tril(g.uniform(-1, 1, (n, n)) / np.sqrt(n), -1) + np.diag(g.uniform(1, 2, n))
    dT = torch.from_numpy(np.ascontiguousarray(T.astype(np.float32).T)).cuda()
    B0 = _rand(g, m, n)
    ws = torch.empty((n // 2) ** 2 + m * n // 2, dtype=torch.float16, device="cuda")
    b1, b2 = B0.clone(), B0.clone()
    _fn(lib, "_Z7tc_trsmP13cublasContextllPflS1_lP6__halfl")(None, m, n, dT.data_ptr(), n, b1.data_ptr(), m,
                                                             ws.data_ptr(), 512)
    tblas._check(lib.tb_strsm(b"R", m, n, dT.data_ptr(), n, b2.data_ptr(), m, 512, 0))
    tblas.synchronize()
    assert torch.equal(b1, b2)
    b1, b2 = B0.clone(), B0.clone()
    _fn(lib, "_Z17tc_cumpsgemm_trsmP13cublasContextPN9cumpsgemm13handle_structEllPflS4_ll")(None, None, m, n, dT.data_ptr(),
                                                                                   n, b1.data_ptr(), m, 512)
    tblas._check(lib.tb_strsm(b"R", m, n, dT.data_ptr(), n, b2.data_ptr(), m, 512, 1))
    tblas.synchronize()
    assert torch.equal(b1, b2)


def test_tc_syr2k_and_cumpsgemm_syr2k(env):
    tblas, g = env
    lib = tblas.lib
    n, k = 900, 640
    A, B, C0 = _rand(g, n, k), _rand(g, n, k), _rand(g, n, n)
    ws = torch.empty(2 * n * k, dtype=torch.float16, device="cuda")
    c1, c2 = C0.clone(), C0.clone()
    _fn(lib, "_Z8tc_syr2kP13cublasContextllfPflS1_lfS1_lP6__halfl")(None, n, k, 1.0, A.data_ptr(), n, B.data_ptr(), n,
                                                                   1.0, c1.data_ptr(), n, ws.data_ptr(), 256)
    tblas._check(lib.tb_ssyr2k(b"L", b"N", n, k, 1.0, A.data_ptr(), n, B.data_ptr(), n, 1.0, c2.data_ptr(), n, 256, 0))
    tblas.synchronize()
    assert torch.equal(c1, c2)
    c1, c2 = C0.clone(), C0.clone()
    _fn(lib, "_Z18tc_cumpsgemm_syr2kPN9cumpsgemm13handle_structEllfPflS2_lfS2_ll")(None, n, k, 1.0, A.data_ptr(), n,
                                                                          B.data_ptr(), n, 1.0, c1.data_ptr(), n, 256)
    tblas._check(lib.tb_ssyr2k(b"L", b"N", n, k, 1.0, A.data_ptr(), n, B.data_ptr(), n, 1.0, c2.data_ptr(), n, 256, 1))
    tblas.synchronize()
    assert torch.equal(c1, c2)


def test_tc_trmm_and_cumpsgemm_trmm(env):
    tblas, g = env
    lib = tblas.lib
    m, n = 1100, 700
    A = torch.tril(_rand(g, m, m).T).T.contiguous()  # lower part only, as the reference requires
    B = _rand(g, m, n)
    ws = torch.empty(m * m + m * n, dtype=torch.float16, device="cuda")
    for name, prec in (("_Z7tc_trmmP13cublasContextllfPflS1_lS1_lP6__halfl", 0),
                       ("_Z17tc_cumpsgemm_trmmPN9cumpsgemm13handle_structEllfPflS2_lS2_ll", 1)):
        c1 = torch.zeros(n, m, device="cuda")
        c2 = torch.zeros_like(c1)
        if prec == 0:
            _fn(lib, name)(None, m, n, 0.75, A.data_ptr(), m, B.data_ptr(), m, c1.data_ptr(), m, ws.data_ptr(), 256)
        else:
            _fn(lib, name)(None, m, n, 0.75, A.data_ptr(), m, B.data_ptr(), m, c1.data_ptr(), m, 256)
        tblas._check(lib.tb_strmm(b"L", m, n, 0.75, A.data_ptr(), m, B.data_ptr(), m, c2.data_ptr(), m, 256, prec))
        tblas.synchronize()
        assert torch.equal(c1, c2), name


def test_tc_symm_and_cumpsgemm_symm(env):
    tblas, g = env
    lib = tblas.lib
    m, n = 1000, 600
    A, B, C0 = _rand(g, m, m), _rand(g, m, n), _rand(g, m, n)
    A_before = A.clone()
    ws = torch.empty(m * m + m * n, dtype=torch.float16, device="cuda")
    for name, prec in (("_Z7tc_symmP13cublasContextllfPflS1_ifS1_lP6__half", 0),
                       ("_Z17tc_cumpsgemm_symmPN9cumpsgemm13handle_structEllfPflS2_ifS2_l", 1)):
        c1, c2 = C0.clone(), C0.clone()
        if prec == 0:
            _fn(lib, name)(None, m, n, 1.25, A.data_ptr(), m, B.data_ptr(), m, -0.5, c1.data_ptr(), m, ws.data_ptr())
        else:
            _fn(lib, name)(None, m, n, 1.25, A.data_ptr(), m, B.data_ptr(), m, -0.5, c1.data_ptr(), m)
        tblas._check(lib.tb_ssymm(b"L", m, n, 1.25, A.data_ptr(), m, B.data_ptr(), m, -0.5, c2.data_ptr(), m, prec))
        tblas.synchronize()
        assert torch.equal(c1, c2), name
    assert torch.equal(A, A_before)  # unlike the reference, A is not symmetrised in place
