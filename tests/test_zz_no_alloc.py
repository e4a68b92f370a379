"""tb_ssyrk_noalloc: the SYRK entry point for callers that cannot allocate.

Callers whose device memory is owned by another allocator, or that cannot
afford the device-wide synchronisation of cudaMalloc/cudaFree, use this
variant; its scratch lives in a static 64 MiB device array inside the
library. The tests call it through the C ABI twice in a row, on different
inputs, and compare each result with the allocating tb_ssyrk on the same
inputs, within the SYRK tolerances of test_gpu_gemm_syrk.py; check in a
fresh process that it makes no device allocation (the library's own
allocation counter stays put and free device memory is unchanged across a
second call); and check that a device-side wait that runs out inside it is
reported by tb_synchronize. This file is named so that pytest collects it
last; it also passes on its own in a fresh process.
"""
import ctypes
import os
import subprocess
import sys
import textwrap

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


@pytest.mark.parametrize("uplo,trans", [(b"U", b"N"), (b"L", b"T")])
def test_noalloc_other_flags_match_allocating_entry_point(tblas, uplo, trans):
    lib = _bind(tblas.lib)
    n, k = 700, 300
    g = np.random.Generator(np.random.PCG64(21))
    rows, cols = (k, n) if trans == b"T" else (n, k)
    A = g.uniform(-1, 1, (rows, cols)).astype(np.float32)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    C0 = torch.from_numpy(g.uniform(-1, 1, (n, n)).astype(np.float32)).cuda()
    c1, c2 = C0.clone(), C0.clone()
    tblas._bind_stream(dA)
    assert lib.tb_ssyrk_noalloc(uplo, trans, n, k, 0.5, dA.data_ptr(), rows, 2.0, c1.data_ptr(), n, 256, 0) == 0
    tblas._check(lib.tb_ssyrk(uplo, trans, n, k, 0.5, dA.data_ptr(), rows, 2.0, c2.data_ptr(), n, 256, 0))
    tblas.synchronize()
    assert torch.equal(c1, c2)
    # nothing to multiply: C = beta C on the triangle, as tb_ssyrk
    assert lib.tb_ssyrk_noalloc(uplo, trans, n, 0, 1.0, dA.data_ptr(), rows, 3.0, c1.data_ptr(), n, 256, 0) == 0
    tblas._check(lib.tb_ssyrk(uplo, trans, n, 0, 1.0, dA.data_ptr(), rows, 3.0, c2.data_ptr(), n, 256, 0))
    tblas.synchronize()
    assert torch.equal(c1, c2)


def test_noalloc_timeout_is_reported_by_synchronize(tblas):
    """A wait that runs out inside the allocation-free SYRK (the test hook
    skips the loads of one tile and shortens the waits to 20 ms) is recorded
    in the call's own static error block and returned by tb_synchronize; the
    next call is correct."""
    lib = _bind(tblas.lib)
    n, k = 600, 256
    g = np.random.Generator(np.random.PCG64(5))
    A = g.uniform(-1, 1, (n, k)).astype(np.float32)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dC = torch.zeros(n, n, device="cuda")
    tblas._bind_stream(dA)
    assert lib.tb_ssyrk_noalloc(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, 256, 0) == 0
    tblas.synchronize()  # the first call has registered the static error block
    tblas._check(lib.tb_debug_stall(0, 20_000_000))
    try:
        assert lib.tb_ssyrk_noalloc(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, 256, 0) == 0
        assert lib.tb_synchronize() == 4  # TB_ERROR_TIMEOUT
    finally:
        lib.tb_debug_stall(-1, 0)
        lib.tb_synchronize()
    assert lib.tb_ssyrk_noalloc(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, 256, 0) == 0
    tblas.synchronize()
    low = np.tril(np.ones((n, n), dtype=bool))
    _, err = orc.rel_errors(dC.cpu().numpy().T, orc.syrk_model(A), low)
    assert err <= _tol(k, 0)


_FRESH = textwrap.dedent("""
    import ctypes, sys
    import torch
    sys.path.insert(0, sys.argv[1])
    import TensorBLAS as T
    lib = T.lib
    n, k = 1000, 700
    A = torch.rand(k, n, device="cuda") * 2 - 1   # column-major n x k
    C = torch.zeros(n, n, device="cuda")
    torch.cuda.synchronize()
    T._bind_stream(A)
    a0 = lib.tb_alloc_count()
    for prec in (0, 1):
        assert lib.tb_ssyrk_noalloc(b"L", b"N", n, k, 1.0, A.data_ptr(), n, 0.0, C.data_ptr(), n, 256, prec) == 0
        assert lib.tb_synchronize() == 0
    a1 = lib.tb_alloc_count()
    free1 = torch.cuda.mem_get_info()[0]
    for prec in (0, 1):
        assert lib.tb_ssyrk_noalloc(b"L", b"N", n, k, 1.0, A.data_ptr(), n, 0.0, C.data_ptr(), n, 256, prec) == 0
        assert lib.tb_synchronize() == 0
    free2 = torch.cuda.mem_get_info()[0]
    a2 = lib.tb_alloc_count()
    print("allocs", a0, a1, a2, "free", free1, free2)
    assert a0 == a1 == a2, (a0, a1, a2)
    assert free1 == free2, (free1, free2)
    print("OK")
""")


def test_noalloc_allocates_nothing_in_a_fresh_process():
    """In a fresh process the allocation-free SYRK is the library's first
    call: the library's allocation counter does not move over its first and
    second calls (both precisions, tb_synchronize included), and free device
    memory is the same before and after the second call."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    py = os.path.join(root, "tensor-blas_b200", "python")
    r = subprocess.run([sys.executable, "-c", _FRESH, py], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
