"""Python front-end of the B200 TensorBLAS library (ctypes over the C ABI).

Mirrors the reference's python/TensorBLAS.py (Orgline/Tensor-BLAS):
``tc_syrk(A, transpose=False, nb=256)`` and ``tc_trsm(A, B, nb=256)`` with the
same argument meaning, the same row-major torch <-> column-major bridging and
the same failure behaviour (``assert status == 0``).  Beyond the reference it
exposes the precision choice and the other BLAS3 routines of include/tb_capi.h.

The shared library is loaded from ../lib/libTensorBLAS.so (built in-tree by
``make -C tensor-blas_b200``); importing this module fails loudly if it is
missing — there is no CPU fallback.
"""
import ctypes
import os

import torch

dir_path = os.path.dirname(os.path.realpath(__file__))
LIB_PATH = os.path.join(dir_path, "..", "lib", "libTensorBLAS.so")
if not os.path.exists(LIB_PATH):
    raise ImportError(f"TensorBLAS native library not built: {LIB_PATH} (run make -C tensor-blas_b200)")
lib = ctypes.CDLL(LIB_PATH)

PLAIN = 0  # FP16 operands, FP32 accumulation (reference tc_*)
SPLIT = 1  # FP16 hi + scaled-lo, 3 products, FP32-level accuracy
FP8 = 2    # e4m3 scaled per 128x128 block (SYRK/SYR2K/TRMM/SYMM/GEMM), ~1e-2 accuracy
REFINE = 3  # TRSM: plain solve + one refinement sweep, FP32-level accuracy
NB_AUTO = -1  # nb for ssyrk / strsm / ssyr2k / strmm: the library's autotuner picks nb and the GEMM engine
# (engine 1: 256 x 256 tiles on CTA pairs, 0: single-CTA 128 x 256, 2: single-CTA 128 x 128, plain only)

_c_long = ctypes.c_long
_fp = ctypes.c_void_p

lib.tc_syrk_wrapper.argtypes = [_c_long, _c_long, _fp, _fp, _c_long]
lib.tc_syrk_wrapper.restype = ctypes.c_int
lib.tc_trsm_wrapper.argtypes = [_c_long, _c_long, _fp, _fp, _c_long]
lib.tc_trsm_wrapper.restype = ctypes.c_int
lib.tb_set_stream.argtypes = [ctypes.c_void_p]
lib.tb_set_stream.restype = ctypes.c_int
lib.tb_synchronize.argtypes = []
lib.tb_synchronize.restype = ctypes.c_int
lib.tb_last_error.argtypes = []
lib.tb_last_error.restype = ctypes.c_char_p
lib.tb_status_string.argtypes = [ctypes.c_int]
lib.tb_status_string.restype = ctypes.c_char_p
lib.tb_launch_count.argtypes = []
lib.tb_launch_count.restype = ctypes.c_ulonglong
lib.tb_profile_begin.argtypes = []
lib.tb_profile_begin.restype = ctypes.c_int
lib.tb_profile_end.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_long)]
lib.tb_profile_end.restype = ctypes.c_int
lib.tb_ssyr2k.argtypes = [ctypes.c_char, ctypes.c_char, _c_long, _c_long, ctypes.c_float, _fp, _c_long, _fp, _c_long,
                          ctypes.c_float, _fp, _c_long, _c_long, ctypes.c_int]
lib.tb_ssyr2k.restype = ctypes.c_int
lib.tb_strmm.argtypes = [ctypes.c_char, _c_long, _c_long, ctypes.c_float, _fp, _c_long, _fp, _c_long, _fp, _c_long,
                         _c_long, ctypes.c_int]
lib.tb_strmm.restype = ctypes.c_int
lib.tb_ssymm.argtypes = [ctypes.c_char, _c_long, _c_long, ctypes.c_float, _fp, _c_long, _fp, _c_long, ctypes.c_float,
                         _fp, _c_long, ctypes.c_int]
lib.tb_ssymm.restype = ctypes.c_int
lib.tb_sgemm.argtypes = [ctypes.c_char, ctypes.c_char, _c_long, _c_long, _c_long, ctypes.c_float, _fp, _c_long, _fp,
                         _c_long, ctypes.c_float, _fp, _c_long, ctypes.c_int]
lib.tb_sgemm.restype = ctypes.c_int
lib.tb_ssyrk.argtypes = [ctypes.c_char, ctypes.c_char, _c_long, _c_long, ctypes.c_float, _fp, _c_long,
                         ctypes.c_float, _fp, _c_long, _c_long, ctypes.c_int]
lib.tb_ssyrk.restype = ctypes.c_int
lib.tb_strsm.argtypes = [ctypes.c_char, _c_long, _c_long, _fp, _c_long, _fp, _c_long, _c_long, ctypes.c_int]
lib.tb_strsm.restype = ctypes.c_int
lib.tb_ssyrk_host.argtypes = lib.tb_ssyrk.argtypes
lib.tb_ssyrk_host.restype = ctypes.c_int
lib.tb_strsm_host.argtypes = lib.tb_strsm.argtypes
lib.tb_autotune_set_file.argtypes = [ctypes.c_char_p]
lib.tb_autotune_set_file.restype = ctypes.c_int
lib.tb_autotune_clear.argtypes = []
lib.tb_autotune_clear.restype = ctypes.c_int
lib.tb_autotune_entries.argtypes = []
lib.tb_autotune_entries.restype = ctypes.c_int
lib.tb_autotune_put.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _c_long, _c_long, ctypes.c_int, _c_long, ctypes.c_int,
                                ctypes.c_double]
lib.tb_autotune_put.restype = ctypes.c_int
lib.tb_autotune_get.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _c_long, _c_long, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_int)]
lib.tb_autotune_get.restype = ctypes.c_int
lib.tb_autotune_put_ex.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _c_long, _c_long, ctypes.c_int, _c_long,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_double]
lib.tb_autotune_put_ex.restype = ctypes.c_int
lib.tb_autotune_get_ex.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _c_long, _c_long, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_int)]
lib.tb_autotune_get_ex.restype = ctypes.c_int
lib.tb_strsm_host.restype = ctypes.c_int
lib.tb_alloc_count.argtypes = []
lib.tb_alloc_count.restype = ctypes.c_ulonglong
lib.tb_release_scratch.argtypes = []
lib.tb_release_scratch.restype = ctypes.c_int
lib.tb_debug_stall.argtypes = [_c_long, ctypes.c_ulonglong]
lib.tb_debug_stall.restype = ctypes.c_int
lib.tb_ssyrk_noalloc.argtypes = lib.tb_ssyrk.argtypes
lib.tb_ssyrk_noalloc.restype = ctypes.c_int


class TensorBLASError(RuntimeError):
    pass


def _check(status):
    if status != 0:
        msg = lib.tb_last_error().decode(errors="replace")
        name = lib.tb_status_string(status).decode()
        raise TensorBLASError(f"{name}: {msg}")


def _bind_stream(t):
    lib.tb_set_stream(ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream))


def _dev_f32(t, name):
    if not (t.is_cuda and t.dtype == torch.float32):
        raise TypeError(f"{name} must be a float32 CUDA tensor")


def _shape(t, name, rows=None, cols=None):
    """A logical matrix argument: 2-D, of the given shape where one is
    required (None: any). A wrong shape would make the kernels read or write
    outside the tensor, so it is an error here, before any device work; the
    callers check every shape first and then every device and dtype
    (`_devs`)."""
    if t.dim() != 2:
        raise ValueError(f"{name} must be a 2-D matrix, got shape {tuple(t.shape)}")
    if (rows is not None and t.shape[0] != rows) or (cols is not None and t.shape[1] != cols):
        want = f"{'*' if rows is None else rows} x {'*' if cols is None else cols}"
        raise ValueError(f"{name} must be {want}, got {t.shape[0]} x {t.shape[1]}")


def _devs(**tensors):
    """Every given tensor (None: an omitted optional argument) is float32 on
    a CUDA device."""
    for name, t in tensors.items():
        if t is not None:
            _dev_f32(t, name)


# ---------------------------------------------------------------- reference API
def tc_syrk(A, transpose=False, nb=256):
    """C = A @ A.T (full symmetric n x n) for a row-major torch A (n x k).

    With transpose=True computes A.T @ A, as python/TensorBLAS.py:11-34.
    """
    _shape(A, "A")
    _devs(A=A)
    if transpose:
        A = torch.clone(A.T).contiguous()
    n = A.size(0)
    k = A.size(1)
    C = torch.zeros(n, n, device=A.device, dtype=torch.float32)
    _bind_stream(A)
    status = lib.tc_syrk_wrapper(n, k, A.data_ptr(), C.data_ptr(), nb)
    assert status == 0
    return C


def tc_trsm(A, B, nb=256):
    """X with X @ A.T = B for lower-triangular A, as python/TensorBLAS.py:43-68."""
    _shape(A, "A")
    n = A.size(0)
    _shape(A, "A", n, n)
    _shape(B, "B", None, n)
    _devs(A=A, B=B)
    m = B.size(0)
    A = torch.clone(A.T).contiguous()
    B_inout = torch.clone(B.T).contiguous()
    _bind_stream(B_inout)
    status = lib.tc_trsm_wrapper(m, n, A.data_ptr(), B_inout.data_ptr(), nb)
    assert status == 0
    return B_inout.T


# ---------------------------------------------------------------- column-major BLAS-style API
# Matrices are passed as torch tensors holding COLUMN-MAJOR data: a tensor
# `T` of shape (cols, rows) row-major is the rows x cols column-major matrix
# T.T. Helpers below take the logical matrix and handle that.
def sgemm(transa, transb, m, n, k, alpha, A_cm, lda, B_cm, ldb, beta, C_cm, ldc, precision=PLAIN):
    """Raw column-major SGEMM on device buffers (tensor-core products at `precision`)."""
    _dev_f32(A_cm, "A")
    _dev_f32(B_cm, "B")
    _dev_f32(C_cm, "C")
    _check(lib.tb_sgemm(transa.encode(), transb.encode(), m, n, k, alpha, A_cm.data_ptr(), lda, B_cm.data_ptr(), ldb,
                        beta, C_cm.data_ptr(), ldc, precision))


def ssyrk(A_cm, C_cm, n, k, lda, ldc, alpha=1.0, beta=0.0, trans="N", nb=256, precision=PLAIN):
    """Raw column-major SSYRK on device buffers (lower triangle)."""
    _dev_f32(A_cm, "A")
    _dev_f32(C_cm, "C")
    _check(lib.tb_ssyrk(b"L", trans.encode(), n, k, alpha, A_cm.data_ptr(), lda, beta, C_cm.data_ptr(), ldc, nb,
                        precision))


def strsm(side, A_cm, B_cm, m, n, lda, ldb, nb=512, precision=PLAIN):
    """Raw column-major STRSM (lower, non-unit); side 'R': X A^T = B, 'L': A X = B."""
    _dev_f32(A_cm, "A")
    _dev_f32(B_cm, "B")
    _check(lib.tb_strsm(side.encode(), m, n, A_cm.data_ptr(), lda, B_cm.data_ptr(), ldb, nb, precision))


def autotune_set_file(path):
    """Keep the autotuner's cache in a JSON file (loaded now, rewritten on
    every new entry); None keeps it in memory only."""
    _check(lib.tb_autotune_set_file(path.encode() if path else None))


def autotune_entries():
    return lib.tb_autotune_entries()


def autotune_get(routine, flags, a, b, precision=PLAIN):
    """The cached (nb, engine) of a key, or None (see tb_autotune_get)."""
    nb, eng = ctypes.c_long(), ctypes.c_int()
    st = lib.tb_autotune_get(routine.encode(), flags.encode(), a, b, precision, ctypes.byref(nb), ctypes.byref(eng))
    return (nb.value, eng.value) if st == 0 else None


def autotune_get_ex(routine, flags, a, b, precision=PLAIN):
    """The cached (nb, engine, split-K parts) of a key, or None (see tb_autotune_get_ex)."""
    nb, eng, sk = ctypes.c_long(), ctypes.c_int(), ctypes.c_int()
    st = lib.tb_autotune_get_ex(routine.encode(), flags.encode(), a, b, precision, ctypes.byref(nb), ctypes.byref(eng),
                                ctypes.byref(sk))
    return (nb.value, eng.value, sk.value) if st == 0 else None


def _host_f32(t, name):
    if t.device.type != "cpu" or t.dtype != torch.float32 or not t.is_contiguous():
        raise TypeError(f"{name} must be a contiguous float32 CPU tensor (page-locked for full speed)")


def ssyrk_host(A_cm, C_cm, n, k, lda, ldc, alpha=1.0, beta=0.0, nb=256, precision=PLAIN):
    """Column-major SSYRK (lower, 'N') with A and C in host memory; the call
    overlaps the copies with the tensor-core work and returns when C is
    written (see tb_ssyrk_host)."""
    _host_f32(A_cm, "A")
    _host_f32(C_cm, "C")
    lib.tb_set_stream(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _check(lib.tb_ssyrk_host(b"L", b"N", n, k, alpha, A_cm.data_ptr(), lda, beta, C_cm.data_ptr(), ldc, nb,
                             precision))


def strsm_host(side, A_cm, B_cm, m, n, lda, ldb, nb=512, precision=PLAIN):
    """Column-major STRSM (lower, non-unit) with A and B in host memory; B is
    overwritten by X (see tb_strsm_host)."""
    _host_f32(A_cm, "A")
    _host_f32(B_cm, "B")
    lib.tb_set_stream(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _check(lib.tb_strsm_host(side.encode(), m, n, A_cm.data_ptr(), lda, B_cm.data_ptr(), ldb, nb, precision))


def syrk(A, alpha=1.0, beta=0.0, C=None, nb=256, precision=PLAIN):
    """Lower triangle of alpha * A @ A.T + beta * C for a logical n x k torch matrix A.

    Returns an n x n tensor whose strict upper triangle is C's (or zero).
    """
    _shape(A, "A")
    n, k = A.shape
    if C is not None:
        _shape(C, "C", n, n)
    _devs(A=A, C=C)
    Acm = A.t().contiguous()  # storage = column-major n x k
    if C is None:
        Ccm = torch.zeros(n, n, device=A.device, dtype=torch.float32)
    else:
        Ccm = C.t().contiguous()
    _bind_stream(A)
    ssyrk(Acm, Ccm, n, k, n, n, alpha, beta, "N", nb, precision)
    return Ccm.t()


def trsm(A, B, side="L", nb=512, precision=PLAIN):
    """Solve A X = B (side 'L') or X A^T = B (side 'R') for lower-triangular A."""
    _shape(B, "B")
    m, n = B.shape
    nt = n if side in ("R", "r") else m
    _shape(A, "A", nt, nt)
    _devs(A=A, B=B)
    Acm = A.t().contiguous()
    Bcm = B.t().contiguous()
    _bind_stream(B)
    strsm(side, Acm, Bcm, m, n, A.shape[0], m, nb, precision)
    return Bcm.t()


def syr2k(A, B, alpha=1.0, beta=0.0, C=None, nb=256, precision=PLAIN):
    """Lower triangle of alpha (A B^T + B A^T) + beta C (logical n x k torch matrices)."""
    _shape(A, "A")
    n, k = A.shape
    _shape(B, "B", n, k)
    if C is not None:
        _shape(C, "C", n, n)
    _devs(A=A, B=B, C=C)
    Acm, Bcm = A.t().contiguous(), B.t().contiguous()
    Ccm = torch.zeros(n, n, device=A.device, dtype=torch.float32) if C is None else C.t().contiguous()
    _bind_stream(A)
    _check(lib.tb_ssyr2k(b"L", b"N", n, k, alpha, Acm.data_ptr(), n, Bcm.data_ptr(), n, beta, Ccm.data_ptr(), n, nb,
                         precision))
    return Ccm.t()


def trmm(A, B, alpha=1.0, uplo="L", nb=256, precision=PLAIN):
    """alpha op(A) B for triangular A ('L' lower / 'U' upper), left side, out of place."""
    _shape(B, "B")
    m, n = B.shape
    _shape(A, "A", m, m)
    _devs(A=A, B=B)
    Acm, Bcm = A.t().contiguous(), B.t().contiguous()
    Ccm = torch.empty(n, m, device=B.device, dtype=torch.float32)
    _bind_stream(B)
    _check(lib.tb_strmm(uplo.encode(), m, n, alpha, Acm.data_ptr(), m, Bcm.data_ptr(), m, Ccm.data_ptr(), m, nb,
                        precision))
    return Ccm.t()


def symm(A, B, alpha=1.0, beta=0.0, C=None, uplo="L", precision=PLAIN):
    """alpha A B + beta C for symmetric A stored in triangle `uplo` (left side)."""
    _shape(B, "B")
    m, n = B.shape
    _shape(A, "A", m, m)
    if C is not None:
        _shape(C, "C", m, n)
    _devs(A=A, B=B, C=C)
    Acm, Bcm = A.t().contiguous(), B.t().contiguous()
    Ccm = torch.zeros(n, m, device=B.device, dtype=torch.float32) if C is None else C.t().contiguous()
    _bind_stream(B)
    _check(lib.tb_ssymm(uplo.encode(), m, n, alpha, Acm.data_ptr(), m, Bcm.data_ptr(), m, beta, Ccm.data_ptr(), m,
                        precision))
    return Ccm.t()


def synchronize():
    _check(lib.tb_synchronize())


def release_scratch():
    """Wait for the device and free the library's scratch pool and cached tile lists."""
    _check(lib.tb_release_scratch())


def alloc_count():
    """Device allocations the library has made in this process."""
    return lib.tb_alloc_count()


# ---------------------------------------------------------------- batched uneven instances
lib.tb_batch_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_void_p),
                                ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_void_p),
                                ctypes.POINTER(ctypes.c_long), ctypes.c_long, ctypes.c_int]
lib.tb_batch_create.restype = ctypes.c_int
lib.tb_batch_run.argtypes = [ctypes.c_void_p]
lib.tb_batch_run.restype = ctypes.c_int
lib.tb_batch_destroy.argtypes = [ctypes.c_void_p]
lib.tb_batch_destroy.restype = ctypes.c_int

SYRK_KIND, TRSM_KIND = 0, 1


class Batch:
    """Many independent SYRK / TRSM instances run by a few grouped launches.

    kinds[i] = SYRK_KIND: C_i(lower) = A_i A_i^T; BC[i] is C_i.
    kinds[i] = TRSM_KIND: X_i A_i^T = B_i with A_i lower; BC[i] is B_i (overwritten).
    A[i], BC[i] are float32 CUDA tensors holding column-major n_i x n_i storage;
    they must stay alive while the batch exists. run() may be captured in a
    CUDA graph.
    """

    def __init__(self, kinds, A, BC, nb=0, precision=SPLIT):
        count = len(kinds)
        if len(A) != count or len(BC) != count:
            raise ValueError("kinds, A and BC need one entry per instance")
        for i, (kind, a, bc) in enumerate(zip(kinds, A, BC)):
            if kind not in (SYRK_KIND, TRSM_KIND):
                raise ValueError(f"kinds[{i}] must be SYRK_KIND or TRSM_KIND")
            side = int(round(a.numel() ** 0.5))
            if side * side != a.numel() or bc.numel() != a.numel():
                raise ValueError(f"A[{i}] and BC[{i}] must both hold one n x n matrix")
        for i, (a, bc) in enumerate(zip(A, BC)):
            _devs(**{f"A[{i}]": a, f"BC[{i}]": bc})
        self._keep = (list(A), list(BC))
        n = [int(round(a.numel() ** 0.5)) for a in A]
        k_arr = (ctypes.c_int * count)(*kinds)
        n_arr = (ctypes.c_long * count)(*n)
        a_arr = (ctypes.c_void_p * count)(*[a.data_ptr() for a in A])
        bc_arr = (ctypes.c_void_p * count)(*[b.data_ptr() for b in BC])
        ld = (ctypes.c_long * count)(*[max(v, 1) for v in n])
        self.handle = ctypes.c_void_p()
        _check(lib.tb_batch_create(ctypes.byref(self.handle), count, k_arr, n_arr, a_arr, ld, bc_arr, ld, nb,
                                   precision))

    def run(self):
        lib.tb_set_stream(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        _check(lib.tb_batch_run(self.handle))

    def close(self):
        if self.handle:
            lib.tb_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
