"""tb_ssyrk_noalloc: the SYRK entry point for callers that cannot allocate.

Callers whose device memory is owned by another allocator, or that cannot
afford the device-wide synchronisation of cudaMalloc/cudaFree, use this
variant; its scratch lives in a static 64 MiB device array inside the
library. The test calls it through the C ABI twice in a row, on different
inputs, and compares each result with the allocating tb_ssyrk on the same
inputs, within the SYRK tolerances of test_gpu_gemm_syrk.py. This file is
named so that pytest collects it last; it also passes on its own in a fresh
process.
"""
import ctypes

import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu


def _bind(lib):
    c = ctypes
    args = [c.c_char, c.c_char, c.c_long, c.c_long, c.c_float, c.c_void_p, c.c_long, c.c_float, c.c_void_p,
            c.c_long, c.c_long, c.c_int]
    lib.tb_ssyrk_noalloc.argtypes = args
    lib.tb_ssyrk_noalloc.restype = c.c_int
    return lib


def _tol(k, precision):
    return 2e-6 if precision else 1e-6 + 1e-8 * k


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_allocating_entry_point_twice(tblas, precision):
    lib = _bind(tblas.lib)
    n, k = 1000, 700
    low = np.tril(np.ones((n, n), dtype=bool))
    for call, seed in enumerate((11, 12)):  # two calls in a row, different inputs
        g = np.random.Generator(np.random.PCG64(seed))
        A = g.uniform(-1, 1, (n, k)).astype(np.float32)
        C0 = g.uniform(-1, 1, (n, n)).astype(np.float32)
        dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
        dC_new = torch.from_numpy(np.ascontiguousarray(C0.T)).cuda()
        dC_ref = dC_new.clone()
        tblas._bind_stream(dA)
        st = lib.tb_ssyrk_noalloc(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.5, dC_new.data_ptr(), n, 256, precision)
        assert st == 0, tblas.lib.tb_last_error()
        tblas._check(lib.tb_ssyrk(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.5, dC_ref.data_ptr(), n, 256, precision))
        tblas.synchronize()
        got = dC_new.cpu().numpy().T
        ref = dC_ref.cpu().numpy().T
        _, err = orc.rel_errors(got, ref, low)
        assert err <= _tol(k, precision), f"call {call}: {err:.3e}"
        assert np.array_equal(got[~low], C0[~low])
        model = orc.syrk_model(A, 1.0, 0.5, C0, split=bool(precision))
        _, err_model = orc.rel_errors(got, model, low)
        assert err_model <= _tol(k, precision), f"call {call} vs oracle: {err_model:.3e}"


def test_noalloc_rejects_oversized_problem(tblas):
    lib = _bind(tblas.lib)
    n, k = 8192, 8192  # FP16 copy of A alone is 128 MiB > 64 MiB
    dA = torch.zeros(1, device="cuda")
    dC = torch.zeros(1, device="cuda")
    st = lib.tb_ssyrk_noalloc(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, 256, 0)
    assert st == 1  # TB_ERROR_INVALID_VALUE, before any device work
    assert b"static maximum" in tblas.lib.tb_last_error()
