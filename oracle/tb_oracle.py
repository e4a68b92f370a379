"""CPU oracle for the TensorBLAS hot path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg (and the
reference arm of bench.py) may import this module, and only to check results
or as the timed CPU baseline; the library never calls it.

It restates, in NumPy, the arithmetic model of the reference's tc_* routines
(Orgline/Tensor-BLAS; paths relative to that project):

* FP32 -> FP16 conversion is round-to-nearest-even (``__float2half`` in
  ``s2h``/``s2h_swpipe``, util/util.cu:127-135, include/TensorBLAS.h:223).
* SYRK (BLAS/tc_syrk.cu:41-157): every product of the recursion is
  FP16 x FP16 with FP32 accumulation over the whole K, so in exact arithmetic
  the plain result is  alpha * h(A) h(A)^T + beta * C  on the lower triangle,
  whatever the chunking.  ``syrk_model`` computes that in FP64.
* TRSM (BLAS/tc_trsm.cu:31-137): solves X A^T = B.  Leaves (n <= nb) are FP32
  ``cublasStrsm``; each internal node converts A21 and B1(=X1) to FP16 and
  applies B2 -= h(X1) h(A21)^T.  In exact arithmetic, with leaf blocks of nb
  columns, X_b = (B_b - sum_{c<b} h(X_c) h(A_bc)^T) A_bb^{-T}.
  ``trsm_right_model`` computes that in FP64.
* The chunk planners find_mat_size_syrk / find_mat_size_trsm
  (util/mat_size.cu:5-55) are restated exactly in ``find_mat_size``.
* The split (error-corrected) form, the role of tc_cumpsgemm_*: operands
  split as hi = h(x), lo = h((x - hi) * 2^11) (Ootomo & Yokota, IJHPCA 2022);
  product = hi*hi + (hi*lo + lo*hi) / 2^11.  ``split_product`` models it.

Parity pin: tests/golden/ holds outputs of the reference library itself
(oracle/_ref/libTensorBLAS_ref.so, built from the reference sources by
oracle/Makefile and run on a B200 by tests/golden/make_golden.py); the tests
check this restatement against those vectors.
"""
from __future__ import annotations

import numpy as np

LO_SCALE = 2048.0  # 2^11


def h(x: np.ndarray) -> np.ndarray:
    """FP32 -> FP16 round-to-nearest-even, returned as FP64 values."""
    return np.asarray(x, dtype=np.float32).astype(np.float16).astype(np.float64)


def split_hilo(x: np.ndarray):
    """hi = h(x); lo = h((x - hi) * 2^11), both as FP64 values (lo unscaled)."""
    x32 = np.asarray(x, dtype=np.float32)
    hi16 = x32.astype(np.float16)
    lo16 = ((x32 - hi16.astype(np.float32)) * np.float32(LO_SCALE)).astype(np.float16)
    return hi16.astype(np.float64), lo16.astype(np.float64)


def split_product(a: np.ndarray, b_t: np.ndarray) -> np.ndarray:
    """Model of the 3-product split GEMM a @ b_t in FP64 arithmetic."""
    ah, al = split_hilo(a)
    bh, bl = split_hilo(b_t)
    return ah @ bh + (ah @ bl + al @ bh) / LO_SCALE


def find_mat_size(n: int, kind: str) -> list[int]:
    """util/mat_size.cu:5-55 — greedy chunk list (the -1 terminator dropped).

    kind "syrk": powers {8192, 16384 x11}, remainder threshold 8192.
    kind "trsm": powers {2048, 4096, 8192, 16384 x8}, threshold 2048.
    """
    if kind == "syrk":
        powers = [8192] + [16384] * 11
        thresh = 8192
    elif kind == "trsm":
        powers = [2048, 4096, 8192] + [16384] * 9
        thresh = 2048
    else:
        raise ValueError(kind)
    out: list[int] = []
    i = len(powers) - 1
    while i >= -1:
        if n < thresh:
            if n != 0:
                out.append(n)
            break
        if i < 0:  # the C loop would index powers[-1] here (n > ~188k)
            raise ValueError("n too large for the reference planner")
        if n >= powers[i]:
            out.append(powers[i])
            n -= powers[i]
        i -= 1
    return out


def syrk_model(A: np.ndarray, alpha: float = 1.0, beta: float = 0.0, C: np.ndarray | None = None,
               trans: bool = False, split: bool = False) -> np.ndarray:
    """Lower triangle (incl. diagonal) of alpha*op(A)op(A)^T + beta*C in FP64.

    A is given as the n x k matrix op(A) (FP32 values).  Upper triangle of the
    result is copied from C (untouched by the routine) or zero.
    """
    A = np.asarray(A, dtype=np.float32)
    if trans:
        A = A.T
    if split:
        prod = split_product(A, A.T)
    else:
        Ah = h(A)
        prod = Ah @ Ah.T
    n = A.shape[0]
    res = alpha * prod
    if C is not None and beta != 0.0:
        res = res + beta * np.asarray(C, dtype=np.float64)
    low = np.tril(np.ones((n, n), dtype=bool))
    base = np.zeros((n, n)) if C is None else np.asarray(C, dtype=np.float64)
    return np.where(low, res, base)


def trsm_right_model(A: np.ndarray, B: np.ndarray, nb: int, split: bool = False) -> np.ndarray:
    """X with X A^T = B (A lower n x n), leaf blocks of nb columns, FP64.

    Off-diagonal block products use FP16-rounded operands (plain) or the
    split model; diagonal blocks are solved exactly (the FP32 leaf).
    """
    A = np.asarray(A, dtype=np.float64)
    B = np.asarray(B, dtype=np.float64)
    m, n = B.shape
    X = np.zeros_like(B)
    blocks = [(s, min(s + nb, n)) for s in range(0, n, nb)]
    for bi, (s, e) in enumerate(blocks):
        R = B[:, s:e].copy()
        for (cs, ce) in blocks[:bi]:
            if split:
                R -= split_product(X[:, cs:ce].astype(np.float32), A[s:e, cs:ce].T.astype(np.float32))
            else:
                R -= h(X[:, cs:ce]) @ h(A[s:e, cs:ce]).T
        # R = X_b A_bb^T  ->  X_b^T = A_bb^{-1} R^T
        X[:, s:e] = np.linalg.solve(A[s:e, s:e], R.T).T
    return X


def trsm_left_model(A: np.ndarray, B: np.ndarray, nb: int, split: bool = False) -> np.ndarray:
    """X with A X = B (A lower m x m): the transpose of the right-side form."""
    return trsm_right_model(A, np.asarray(B).T, nb, split).T


def rel_errors(x: np.ndarray, ref: np.ndarray, mask: np.ndarray | None = None):
    """(max elementwise relative, normwise relative) error of x vs ref."""
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if mask is not None:
        x = x[mask]
        ref = ref[mask]
    d = np.abs(x - ref)
    scale = np.maximum(np.abs(ref), np.finfo(np.float64).tiny)
    nrm = np.linalg.norm(ref)
    return float(np.max(d / scale)) if d.size else 0.0, float(np.linalg.norm(d) / nrm) if nrm > 0 else 0.0


def _prod(a, b_t, split):
    """a @ b_t with FP16-rounded operands (plain) or the split model."""
    if split:
        return split_product(np.asarray(a, np.float32), np.asarray(b_t, np.float32))
    return h(a) @ h(b_t)


def syr2k_model(A, B, alpha=1.0, beta=0.0, C=None, split=False):
    """Lower triangle of alpha (A B^T + B A^T) + beta C (BLAS/tc_syr2k.cu:3-34):
    each product FP16 x FP16 with FP32 accumulation, evaluated exactly."""
    A = np.asarray(A, np.float32)
    B = np.asarray(B, np.float32)
    n = A.shape[0]
    res = alpha * (_prod(A, B.T, split) + _prod(B, A.T, split))
    if C is not None and beta != 0.0:
        res = res + beta * np.asarray(C, np.float64)
    low = np.tril(np.ones((n, n), dtype=bool))
    base = np.zeros((n, n)) if C is None else np.asarray(C, np.float64)
    return np.where(low, res, base)


def trmm_model(A, B, alpha=1.0, upper=False, split=False):
    """alpha op(A) B with A triangular (BLAS/tc_trmm.cu:4-98); the other
    triangle of A is treated as zero."""
    A = np.asarray(A, np.float32)
    T = np.triu(A) if upper else np.tril(A)
    return alpha * _prod(T, np.asarray(B, np.float32), split)


def symm_model(A, B, alpha=1.0, beta=0.0, C=None, lower=True, split=False):
    """alpha A B + beta C with A symmetric from its stored triangle
    (BLAS/tc_symm.cu:3-19)."""
    A = np.asarray(A, np.float32)
    S = np.tril(A) + np.tril(A, -1).T if lower else np.triu(A) + np.triu(A, 1).T
    res = alpha * _prod(S, np.asarray(B, np.float32), split)
    if C is not None and beta != 0.0:
        res = res + beta * np.asarray(C, np.float64)
    return res


# ------------------------------------------------------------------ Ozaki INT8 scheme
def ozaki_slices(A, S):
    """Exact slicing used for the INT8 emulation of FP64 products.

    e_i = frexp exponent of max_p |a_ip| (so |a_ip| < 2^e_i; 0 for a zero
    row); x = a * 2^-e_i; for each slice y = 128 x, q = trunc(y), x = y - q.
    Returns (Q int8 [S, n, k], e int [n]). Every step is exact in FP64.
    """
    A = np.asarray(A, dtype=np.float64)
    _, e = np.frexp(np.max(np.abs(A), axis=1) if A.size else np.zeros(A.shape[0]))
    e = e.astype(np.int64)
    x = np.ldexp(A, -e[:, None])
    Q = np.empty((S,) + A.shape, dtype=np.int8)
    for s in range(S):
        y = x * 128.0
        q = np.trunc(y)
        x = y - q
        Q[s] = q.astype(np.int8)
    return Q, e


def ozaki_level_product(Q, L):
    """P_L = sum_{s+t=L} Q_s Q_t^T in exact int64 (slices numbered from 1)."""
    S = Q.shape[0]
    P = np.zeros((Q.shape[1], Q.shape[1]), dtype=np.int64)
    for s in range(max(1, L - S), min(S, L - 1) + 1):
        P += Q[s - 1].astype(np.int64) @ Q[L - s - 1].astype(np.int64).T
    return P


def ozaki_syrk_model(A, S):
    """The truncated Ozaki sum C = sum_{L=2}^{S+1} 2^(e_i+e_j-7L) P_L (long double)."""
    Q, e = ozaki_slices(A, S)
    n = Q.shape[1]
    C = np.zeros((n, n), dtype=np.longdouble)
    scale = np.ldexp(np.longdouble(1.0), (e[:, None] + e[None, :]).astype(np.int64))
    for L in range(2, S + 2):
        C += ozaki_level_product(Q, L).astype(np.longdouble) * scale * np.ldexp(np.longdouble(1.0), -7 * L)
    return C


def ozaki_gemm_model(A, B, S):
    """The truncated Ozaki product of A (M x K) and B^T (B: N x K), each row
    sliced under its own exponent: sum_{L=2}^{S+1} 2^(eA_i+eB_j-7L) P_L with
    P_L = sum_{s+t=L} QA_s QB_t^T (long double). The FP64 SYR2K/TRMM/TRSM
    products of the INT8 engine are this sum (per K chunk), folded in FP64."""
    QA, ea = ozaki_slices(A, S)
    QB, eb = ozaki_slices(B, S)
    C = np.zeros((QA.shape[1], QB.shape[1]), dtype=np.longdouble)
    scale = np.ldexp(np.longdouble(1.0), (ea[:, None] + eb[None, :]).astype(np.int64))
    for L in range(2, S + 2):
        P = np.zeros(C.shape, dtype=np.int64)
        for s in range(max(1, L - S), min(S, L - 1) + 1):
            P += QA[s - 1].astype(np.int64) @ QB[L - s - 1].astype(np.int64).T
        C += P.astype(np.longdouble) * scale * np.ldexp(np.longdouble(1.0), -7 * L)
    return C


def gemm_extended(A, B):
    """A B^T in long double (64-bit mantissa); A M x K, B N x K."""
    return np.asarray(A, np.float64).astype(np.longdouble) @ np.asarray(B, np.float64).astype(np.longdouble).T


def syrk_extended(A, rows, cols):
    """Entries (rows[i], cols[i]) of A A^T in long double (64-bit mantissa):
    the higher-than-FP64 oracle for the FP64-emulation checks."""
    Al = np.asarray(A, dtype=np.float64).astype(np.longdouble)
    return np.einsum("ij,ij->i", Al[rows], Al[cols])


def e4m3(y):
    """Round float values to FP8 e4m3 (round to nearest even, saturating at
    +-448; normal exponents -6..8, subnormal step 2^-9), as float64."""
    y = np.asarray(y, dtype=np.float64)
    a = np.abs(y)
    _, E = np.frexp(np.where(a > 0, a, 1.0))
    e = np.maximum(E - 1, -6)                  # exponent of the binade (subnormals share -6)
    step = np.ldexp(1.0, e - 3)                # 3 stored mantissa bits
    q = np.round(a / step) * step              # numpy rounds half to even
    q = np.minimum(q, 448.0)
    return np.where(a > 0, np.sign(y) * q, 0.0)


def fp8_quantize(X, block=128):
    """Per-(128-row, 128-deep) block scaled e4m3 copy of an operand X (rows x
    K, row i = one K-vector): s = float32(max|x| / 448) (1 for an all-zero
    block), q = e4m3(float32(x / s)). Returns (Q float64 rows x K, S [rb, kb])."""
    X = np.asarray(X, dtype=np.float32)
    rows, K = X.shape
    rb, kb = -(-rows // block), -(-K // block)
    Q = np.zeros((rows, K))
    S = np.ones((rb, kb), dtype=np.float32)
    for i in range(rb):
        for j in range(kb):
            blk = X[i * block:(i + 1) * block, j * block:(j + 1) * block]
            m = np.float32(np.max(np.abs(blk))) if blk.size else np.float32(0)
            s = np.float32(m / np.float32(448.0)) if m > 0 else np.float32(1.0)
            S[i, j] = s
            Q[i * block:(i + 1) * block, j * block:(j + 1) * block] = e4m3((blk / s).astype(np.float32))
    return Q, S


def fp8_product_model(A, B, block=128):
    """sum over 128-deep K blocks of s_A s_B (Q_A Q_B^T) for A (M x K) and
    B (N x K), in float64: what the FP8 engine computes before rounding."""
    QA, SA = fp8_quantize(A, block)
    QB, SB = fp8_quantize(B, block)
    M, K = QA.shape
    N = QB.shape[0]
    C = np.zeros((M, N))
    for kb in range(SA.shape[1]):
        ks = slice(kb * block, (kb + 1) * block)
        P = QA[:, ks] @ QB[:, ks].T
        sa = np.repeat(SA[:, kb].astype(np.float64), block)[:M]
        sb = np.repeat(SB[:, kb].astype(np.float64), block)[:N]
        C += P * sa[:, None] * sb[None, :]
    return C
