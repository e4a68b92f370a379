"""The host-side FP32 -> FP16 conversion (tb_host_s2h, used by the
host-memory SYRK before A crosses PCIe) is bit-exact against NumPy's
round-to-nearest-even float16 conversion: random values over the whole
half range and beyond, every tie between neighbouring halves (normal and
subnormal), the overflow boundary, signed zeros, infinities, strided
operands (leading dimensions larger than the rows) and ragged sizes that
leave a tail after the eight-wide vector path; the same checks again with
the portable bit-level path forced (TB_HOST_F16C=0, in a subprocess). Runs
on the CPU."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import TensorBLAS as TB

L, P = ctypes.c_long, ctypes.c_void_p
TB.lib.tb_host_s2h.argtypes = [L, L, P, L, P, L]
TB.lib.tb_host_s2h.restype = ctypes.c_int


def _convert(A, rows, cols, lda, ldd):
    """A: column-major rows x cols with leading dimension lda (numpy float32, Fortran layout of a lda x cols array)."""
    out = np.full((cols, ldd), 0x7E00, dtype=np.uint16)  # column-major storage: out[j, i]
    src = np.ascontiguousarray(A.T)  # src[j, i] = A[i, j], lda == A.shape[0]
    assert TB.lib.tb_host_s2h(rows, cols, src.ctypes.data_as(P), lda, out.ctypes.data_as(P), ldd) == 0
    return out


def _expect(vals):
    with np.errstate(over="ignore"):
        return vals.astype(np.float16).view(np.uint16)


@pytest.mark.parametrize("rows,cols,lda,ldd", [(1000, 7, 1000, 1000), (37, 513, 40, 64), (8, 1, 8, 8),
                                               (1024, 300, 1030, 1032)])
def test_random_values_bit_exact(rows, cols, lda, ldd):
    g = np.random.Generator(np.random.PCG64(rows * 31 + cols))
    mag = np.exp2(g.uniform(-30, 18, (lda, cols)))
    A = (mag * g.choice([-1.0, 1.0], (lda, cols))).astype(np.float32)
    out = _convert(A, rows, cols, lda, ldd)
    for j in range(cols):
        np.testing.assert_array_equal(out[j, :rows], _expect(A[:rows, j]))
        assert np.all(out[j, rows:] == 0x7E00)  # padding rows untouched


def test_ties_boundaries_and_specials():
    h = np.arange(0, 0x7C00, dtype=np.uint32)  # every finite non-negative half
    lo = h.astype(np.uint16).view(np.float16).astype(np.float32)
    hi = (h + 1).astype(np.uint16).view(np.float16).astype(np.float32)
    mid = ((lo.astype(np.float64) + hi.astype(np.float64)) / 2).astype(np.float32)  # exact: halves have 11 bits
    near = np.nextafter(mid, np.float32(np.inf))
    below = np.nextafter(mid, np.float32(0))
    special = np.array([0.0, -0.0, np.inf, -np.inf, 65504.0, 65519.996, 65520.0, 65536.0, 1e30, -1e30,
                        2.0 ** -24, 2.0 ** -25, np.nextafter(np.float32(2.0 ** -25), np.float32(1)), 2.0 ** -26,
                        2.0 ** -14, np.nextafter(np.float32(2.0 ** -14), np.float32(0)), 1e-45, -1e-45],
                       dtype=np.float32)
    vals = np.concatenate([lo, mid, near, below, -mid, -near, special]).astype(np.float32)
    n = len(vals)
    out = _convert(vals.reshape(n, 1), n, 1, n, n)
    np.testing.assert_array_equal(out[0], _expect(vals))


def test_nan_stays_nan():
    vals = np.array([np.nan, -np.nan] * 8, dtype=np.float32)
    out = _convert(vals.reshape(16, 1), 16, 1, 16, 16)
    h = out[0]
    assert np.all((h & 0x7C00) == 0x7C00) and np.all((h & 0x03FF) != 0)


def test_rejects_bad_arguments():
    buf = np.zeros(16, dtype=np.float32)
    dst = np.zeros(16, dtype=np.uint16)
    assert TB.lib.tb_host_s2h(4, 2, buf.ctypes.data_as(P), 3, dst.ctypes.data_as(P), 4) != 0  # lda < m
    assert TB.lib.tb_host_s2h(4, 2, buf.ctypes.data_as(P), 4, dst.ctypes.data_as(P), 3) != 0  # ldd < m
    assert TB.lib.tb_host_s2h(0, 2, None, 1, None, 1) == 0


def test_portable_path_bit_exact():
    """Every test above with the F16C instructions switched off."""
    env = dict(os.environ, TB_HOST_F16C="0")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", os.path.abspath(__file__),
                        "-k", "not portable"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
