"""CPU checks of the persistent TRSM solve's task plan (tb_debug_trsm_plan,
host only): for every shape the claim order is topological — each task's
waits are met by tasks claimed before it, which is what makes the
persistent kernel deadlock-free whatever the timing — and every tile, K
range and counter index lies inside its op and its arrays."""
import ctypes
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tensor-blas_b200", "lib", "libTensorBLAS.so")


@pytest.fixture(scope="module")
def lib():
    lib = ctypes.CDLL(LIB)
    lib.tb_debug_trsm_plan.argtypes = [ctypes.c_char, ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_long)]
    lib.tb_last_error.restype = ctypes.c_char_p
    return lib


@pytest.mark.parametrize("side,m,n,nb,prec", [
    (b"L", 16384, 16384, 512, 0), (b"R", 16384, 16384, 512, 0), (b"L", 16384, 16384, 512, 1),
    (b"L", 2048, 3000, 512, 0), (b"R", 2900, 2048, 512, 0), (b"L", 2500, 1300, 512, 0),
    (b"R", 700, 2500, 256, 1), (b"L", 4096, 4096, 256, 1), (b"L", 1536, 1000, 512, 0),
    (b"L", 8192, 100, 128, 0), (b"R", 33, 5000, 512, 1), (b"L", 1088, 64, 64, 0),
])
def test_plan_is_topological_and_in_range(lib, side, m, n, nb, prec):
    stats = (ctypes.c_long * 4)()
    st = lib.tb_debug_trsm_plan(side, m, n, nb, prec, stats)
    assert st == 0, lib.tb_last_error()
    tasks, counters, ops, makespan = list(stats)
    nt = m if side == b"L" else n
    leaf = min(512, -(-nb // 64) * 64)
    leaves = -(-nt // leaf)
    assert ops == 2 * leaves - 1  # one product per leaf, one update per internal node
    assert tasks > 0 and counters > 0 and makespan > 0


def test_plan_rejects_bad_arguments(lib):
    stats = (ctypes.c_long * 4)()
    assert lib.tb_debug_trsm_plan(b"X", 10, 10, 64, 0, stats) == 1
    assert lib.tb_debug_trsm_plan(b"L", 0, 10, 64, 0, stats) == 1
