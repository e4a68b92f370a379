"""CPU port of the reference's plain SYRK/TRSM method — TEST INFRASTRUCTURE.

Timed by bench.py as the CPU baseline (``cpu_baseline.kind = "port"``) and by
its reference arm when the reference library is unavailable; never part of
the product. The arithmetic follows the reference (BLAS/tc_syrk.cu:62-125,
BLAS/tc_trsm.cu:31-137): operands rounded FP32 -> FP16 (round-to-nearest),
products accumulated in FP32 — here with the host's FP32 BLAS (OpenBLAS via
SciPy) on all cores — and FP32 triangular solves for the diagonal blocks.
"""
from __future__ import annotations

import os
import time

import numpy as np
from scipy.linalg import blas


def _h32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float16).astype(np.float32)


def syrk_plain(A: np.ndarray) -> np.ndarray:
    """Lower triangle of h(A) h(A)^T with FP32 accumulation (A n x k, Fortran order)."""
    Ah = np.asfortranarray(_h32(A))
    return blas.ssyrk(1.0, Ah, lower=1)


def trsm_left_plain(A: np.ndarray, B: np.ndarray, nb: int) -> np.ndarray:
    """A X = B (A lower m x m) by recursive halving with FP16-operand updates."""
    X = np.asfortranarray(np.array(B, dtype=np.float32))
    A = np.asfortranarray(np.asarray(A, dtype=np.float32))

    def rec(s, e):
        if e - s <= nb:
            X[s:e] = blas.strsm(1.0, A[s:e, s:e], X[s:e], lower=1)
            return
        mid = s + (((e - s + nb - 1) // nb + 1) // 2) * nb
        rec(s, mid)
        X[mid:e] -= _h32(A[mid:e, s:mid]) @ _h32(X[s:mid])
        rec(mid, e)

    rec(0, A.shape[0])
    return X


def threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def time_step(n: int, min_seconds: float = 10.0, seed: int = 0):
    """Repeat (SYRK n=k=n, TRSM m=n=n) until min_seconds; returns (flops/s, reps)."""
    from threadpoolctl import threadpool_limits

    g = np.random.Generator(np.random.PCG64(seed))
    A = np.asfortranarray(g.uniform(-1, 1, (n, n)).astype(np.float32))
    T = np.asfortranarray((np.tril(g.uniform(-1, 1, (n, n)) / np.sqrt(n), -1)
                           + np.diag(g.uniform(1, 2, n))).astype(np.float32))
    B = np.asfortranarray(g.uniform(-1, 1, (n, n)).astype(np.float32))
    with threadpool_limits(threads()):
        syrk_plain(A)  # warm-up
        reps, t0 = 0, time.perf_counter()
        while True:
            syrk_plain(A)
            trsm_left_plain(T, B, 512)
            reps += 1
            el = time.perf_counter() - t0
            if el >= min_seconds:
                break
    return reps * 2.0 * float(n) ** 3 / el, reps, el


def host_blas_rates(n: int = 4096, min_seconds: float = 2.0, seed: int = 1) -> dict:
    """Host BLAS (OpenBLAS via SciPy, all cores) on the level-3 routines this
    library replaces: SSYRK/DSYRK (lower, n = k), STRSM (left, lower,
    non-unit), STRMM (left, upper) and SSYMM (left, lower), all n x n.
    Returns {routine: TFLOP/s} at the nominal BLAS3 flop counts (SYRK, TRSM
    and TRMM n^3, SYMM 2 n^3), each repeated for min_seconds."""
    from threadpoolctl import threadpool_limits

    g = np.random.Generator(np.random.PCG64(seed))
    A = np.asfortranarray(g.uniform(-1, 1, (n, n)).astype(np.float32))
    B = np.asfortranarray(g.uniform(-1, 1, (n, n)).astype(np.float32))
    T = np.asfortranarray((np.tril(g.uniform(-1, 1, (n, n)) / np.sqrt(n), -1)
                           + np.diag(g.uniform(1, 2, n))).astype(np.float32))
    A64 = np.asfortranarray(A.astype(np.float64))
    nf = float(n) ** 3
    cases = {
        "ssyrk": (lambda: blas.ssyrk(1.0, A, lower=1), nf),
        "dsyrk": (lambda: blas.dsyrk(1.0, A64, lower=1), nf),
        "strsm": (lambda: blas.strsm(1.0, T, B, lower=1), nf),
        "strmm": (lambda: blas.strmm(1.0, T.T, B, lower=0), nf),
        "ssymm": (lambda: blas.ssymm(1.0, A, B, lower=1), 2.0 * nf),
    }
    out = {}
    with threadpool_limits(threads()):
        for name, (fn, fl) in cases.items():
            fn()  # warm-up
            reps, t0 = 0, time.perf_counter()
            while True:
                fn()
                reps += 1
                el = time.perf_counter() - t0
                if el >= min_seconds:
                    break
            out[name] = reps * fl / el / 1e12
    return out
