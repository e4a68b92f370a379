"""Bit-exact check of the FP32 -> FP16 conversion kernels (tb_s2h, the
library's replacement of the reference's s2h, util/util.cu:127-136) against
NumPy's round-to-nearest-even float16 cast: hi = fp16(x) and the split form's
lo = fp16((x - hi) * 2^11), on values chosen to hit every rounding case —
exact ties (to even, both directions), the subnormal range and its ties,
the underflow to zero, the largest finite values and the overflow to
infinity, signed zeros — plus wide-exponent random data. Both kernels are
covered: the 8-wide vector path (rows a multiple of 8, aligned) and the
scalar path (ragged rows, odd leading dimension)."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _special_values():
    f16 = np.arange(0, 0x7C00, dtype=np.uint16).view(np.float16).astype(np.float32)  # every finite fp16 >= 0
    nxt = np.nextafter(f16.astype(np.float16), np.float16(np.inf)).astype(np.float32)
    mid = (f16.astype(np.float64) + nxt.astype(np.float64)) / 2           # exact ties (representable in fp32)
    mid = mid[np.isfinite(mid)].astype(np.float32)
    up = np.nextafter(mid, np.float32(np.inf))
    dn = np.nextafter(mid, np.float32(-np.inf))
    extra = np.array([0.0, 2.0 ** -25, 2.0 ** -26, 3 * 2.0 ** -26, 2.0 ** -24 * 1.5, 65504.0, 65519.99, 65520.0,
                      1e6, 3.4e38, 1e-30], dtype=np.float32)
    v = np.concatenate([f16, mid, up, dn, extra])
    return np.concatenate([v, -v])


def _model(x, scale):
    hi = x.astype(np.float16)
    with np.errstate(invalid="ignore", over="ignore"):
        lo = ((x - hi.astype(np.float32)) * np.float32(scale)).astype(np.float16)
    return hi, lo


@pytest.mark.parametrize("rows,ld", [(1024, 1024), (1000, 1003)])  # vector path; scalar path
def test_s2h_bit_exact_vs_numpy(tblas, rows, ld):
    lib = tblas.lib
    lib.tb_s2h.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
                           ctypes.c_long, ctypes.c_void_p, ctypes.c_float]
    g = np.random.Generator(np.random.PCG64(8))
    sv = _special_values()
    wide = (g.standard_normal(200_000) * np.exp2(g.uniform(-30, 20, 200_000))).astype(np.float32)
    vals = np.concatenate([sv, wide])
    cols = -(-vals.size // rows)
    vals = np.concatenate([vals, np.zeros(rows * cols - vals.size, np.float32)])
    g.shuffle(vals)
    X = np.zeros((cols, ld), np.float32)          # column-major rows x cols, leading dimension ld
    X[:, :rows] = vals.reshape(cols, rows)
    dX = torch.from_numpy(X).cuda()
    dH = torch.zeros(cols, ld, dtype=torch.float16, device="cuda")
    dL = torch.zeros_like(dH)
    tblas._bind_stream(dX)
    tblas._check(lib.tb_s2h(rows, cols, dX.data_ptr(), ld, dH.data_ptr(), ld, dL.data_ptr(), 2048.0))
    tblas.synchronize()
    hi, lo = _model(X[:, :rows], 2048.0)
    got_hi = dH.cpu().numpy()[:, :rows].view(np.uint16)
    got_lo = dL.cpu().numpy()[:, :rows].view(np.uint16)
    assert np.array_equal(got_hi, hi.view(np.uint16))
    assert np.array_equal(got_lo, lo.view(np.uint16))
    # the plain form (no lo) writes the same hi
    dH2 = torch.zeros_like(dH)
    tblas._check(lib.tb_s2h(rows, cols, dX.data_ptr(), ld, dH2.data_ptr(), ld, None, 2048.0))
    tblas.synchronize()
    assert torch.equal(dH2[:, :rows].view(torch.int16), dH[:, :rows].view(torch.int16))
