"""Records outputs of the REFERENCE library on seeded inputs (run on a B200).

    make -C oracle                      # builds oracle/_ref/ from the reference sources
    python tests/golden/make_golden.py  # writes tests/golden/ref_*.npz

The reference routines run through oracle/_ref/libTensorBLAS_ref.so
(oracle/ref_driver.cu wraps the reference's own tc_* C++ API with host
buffers). Large outputs are stored as sampled entries plus row sums.
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
import golden_inputs as gi  # noqa: E402

lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libTensorBLAS_ref.so"))
P = ctypes.c_void_p
L = ctypes.c_long
lib.ref_syrk.argtypes = [L, L, ctypes.c_float, P, ctypes.c_float, P, L]
lib.ref_trsm.argtypes = [L, L, P, P, L]
lib.ref_trmm.argtypes = [L, L, ctypes.c_float, P, P, P, L]
lib.ref_syr2k.argtypes = [L, L, ctypes.c_float, P, P, ctypes.c_float, P, L]
lib.ref_symm.argtypes = [L, L, ctypes.c_float, P, P, ctypes.c_float, P]
lib.ref_ozimmu_syrk.argtypes = [L, L, ctypes.c_double, P, ctypes.c_double, P, L]
lib.ref_ozimmu_trsm.argtypes = [L, L, P, P, L]
lib.ref_ozimmu_trmm.argtypes = [L, L, ctypes.c_double, P, P, P, L]
lib.ref_ozimmu_syr2k.argtypes = [L, L, ctypes.c_double, P, P, ctypes.c_double, P, L]
for f in ("ref_syrk", "ref_trsm", "ref_trmm", "ref_syr2k", "ref_symm", "ref_ozimmu_syrk", "ref_ozimmu_trsm",
          "ref_ozimmu_trmm", "ref_ozimmu_syr2k"):
    getattr(lib, f).restype = ctypes.c_int


def cm(x):
    """Column-major (Fortran) copy and its pointer."""
    a = np.asfortranarray(x)
    return a, a.ctypes.data_as(P)


def save(name, **kw):
    np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), **kw)
    print("wrote", name, {k: getattr(v, "shape", v) for k, v in kw.items()})


def sample_lower(n, count, seed):
    g = gi.rng(seed)
    i = g.integers(0, n, count)
    j = g.integers(0, n, count)
    lo, hi = np.maximum(i, j), np.minimum(i, j)
    return lo, hi


def syrk(name, n, k, nb, alpha, beta, seed, full):
    A = gi.uniform(seed, (n, k))
    C0 = gi.uniform(seed + 1, (n, n)) if beta != 0 else np.zeros((n, n), np.float32)
    Af, pA = cm(A)
    Cf, pC = cm(C0)
    assert lib.ref_syrk(n, k, alpha, pA, beta, pC, nb) == 0
    meta = dict(n=n, k=k, nb=nb, alpha=alpha, beta=beta, seed=seed, a_sum=gi.checksum(A))
    if full:
        save(name, C=np.tril(Cf).astype(np.float32), meta=json.dumps(meta))
    else:
        rows, cols = sample_lower(n, 20000, seed + 2)
        save(name, rows=rows, cols=cols, vals=Cf[rows, cols].astype(np.float32),
             rowsum=np.tril(Cf).astype(np.float64).sum(axis=1), meta=json.dumps(meta))


def trsm(name, m, n, nb, seed):
    A = gi.lower_tri(seed, n)
    B = gi.uniform(seed + 1, (m, n))
    Af, pA = cm(A)
    Bf, pB = cm(B)
    assert lib.ref_trsm(m, n, pA, pB, nb) == 0
    save(name, X=Bf.astype(np.float32), meta=json.dumps(dict(m=m, n=n, nb=nb, seed=seed)))


def syr2k(name, n, k, nb, seed, full):
    A = gi.uniform(seed, (n, k))
    B = gi.uniform(seed + 1, (n, k))
    C0 = np.zeros((n, n), np.float32)
    Af, pA = cm(A)
    Bf, pB = cm(B)
    Cf, pC = cm(C0)
    assert lib.ref_syr2k(n, k, 1.0, pA, pB, 0.0, pC, nb) == 0
    meta = json.dumps(dict(n=n, k=k, nb=nb, seed=seed))
    if full:
        save(name, C=np.tril(Cf).astype(np.float32), meta=meta)
    else:
        rows, cols = sample_lower(n, 20000, seed + 2)
        save(name, rows=rows, cols=cols, vals=Cf[rows, cols].astype(np.float32), meta=meta)


def trmm(name, m, n, nb, seed):
    A = np.tril(gi.uniform(seed, (m, m)))  # the reference needs a zero upper triangle
    B = gi.uniform(seed + 1, (m, n))
    Af, pA = cm(A)
    Bf, pB = cm(B)
    Cf, pC = cm(np.zeros((m, n), np.float32))
    assert lib.ref_trmm(m, n, 1.0, pA, pB, pC, nb) == 0
    save(name, C=Cf.astype(np.float32), meta=json.dumps(dict(m=m, n=n, nb=nb, seed=seed)))


def symm(name, m, seed):
    A = gi.uniform(seed, (m, m))
    B = gi.uniform(seed + 1, (m, m))
    Af, pA = cm(A)
    Bf, pB = cm(B)
    Cf, pC = cm(np.zeros((m, m), np.float32))
    assert lib.ref_symm(m, m, 1.0, pA, pB, 0.0, pC) == 0
    save(name, C=Cf.astype(np.float32), meta=json.dumps(dict(m=m, seed=seed)))


def ozimmu_syrk(name, n, k, nb, seed, phi):
    g = gi.rng(seed)
    A = g.standard_normal((n, k)) * np.exp(phi * g.standard_normal((n, k)))
    Af, pA = cm(A)
    Cf, pC = cm(np.zeros((n, n)))
    assert lib.ref_ozimmu_syrk(n, k, 1.0, pA, 0.0, pC, nb) == 0
    save(name, C=np.tril(Cf), meta=json.dumps(dict(n=n, k=k, nb=nb, seed=seed, phi=phi)))


def ozimmu_trsm(name, m, n, nb, seed):
    A = gi.lower_tri(seed, n).astype(np.float64)
    B = gi.rng(seed + 1).uniform(-1, 1, (m, n))
    Af, pA = cm(A)
    Bf, pB = cm(B)
    assert lib.ref_ozimmu_trsm(m, n, pA, pB, nb) == 0
    save(name, X=Bf, meta=json.dumps(dict(m=m, n=n, nb=nb, seed=seed)))


def ozimmu_trmm(name, m, n, nb, seed):
    g = gi.rng(seed)
    A = np.tril(g.standard_normal((m, m)))  # the reference needs a zero upper triangle
    B = g.standard_normal((m, n))
    Af, pA = cm(A)
    Bf, pB = cm(B)
    Cf, pC = cm(np.zeros((m, n)))
    assert lib.ref_ozimmu_trmm(m, n, 1.0, pA, pB, pC, nb) == 0
    save(name, C=Cf, meta=json.dumps(dict(m=m, n=n, nb=nb, seed=seed)))


def ozimmu_syr2k(name, n, k, nb, seed):
    g = gi.rng(seed)
    A = g.standard_normal((n, k))
    B = g.standard_normal((n, k))
    Af, pA = cm(A)
    Bf, pB = cm(B)
    Cf, pC = cm(np.zeros((n, n)))
    assert lib.ref_ozimmu_syr2k(n, k, 1.0, pA, pB, 0.0, pC, nb) == 0
    save(name, C=np.tril(Cf), meta=json.dumps(dict(n=n, k=k, nb=nb, seed=seed)))


FIXTURES = {
    "syrk_small": lambda: syrk("syrk_small", 256, 128, 64, 1.0, 0.0, 101, True),
    "syrk_beta": lambda: syrk("syrk_beta", 200, 50, 64, 0.5, 2.0, 202, True),
    "syrk_p2": lambda: syrk("syrk_p2", 8192, 64, 256, 1.0, 0.0, 303, False),
    "trsm_p2": lambda: trsm("trsm_p2", 64, 2048, 256, 404),
    "trsm_small": lambda: trsm("trsm_small", 64, 1000, 256, 505),
    "trsm_p2_nb512": lambda: trsm("trsm_p2_nb512", 32, 4096, 512, 606),
    "syr2k_small": lambda: syr2k("syr2k_small", 256, 64, 64, 707, True),
    "syr2k_p2": lambda: syr2k("syr2k_p2", 8192, 32, 256, 808, False),
    "trmm_small": lambda: trmm("trmm_small", 256, 128, 64, 909),
    "trmm_p2": lambda: trmm("trmm_p2", 8192, 16, 256, 1010),
    "symm_small": lambda: symm("symm_small", 256, 1111),
    "dsyrk_small": lambda: ozimmu_syrk("dsyrk_small", 256, 128, 64, 1212, 0.5),
    "dtrsm_small": lambda: ozimmu_trsm("dtrsm_small", 192, 2048, 256, 1313),
    "dtrmm_small": lambda: ozimmu_trmm("dtrmm_small", 512, 96, 64, 1414),
    "dsyr2k_small": lambda: ozimmu_syr2k("dsyr2k_small", 384, 200, 64, 1515),
}

if __name__ == "__main__":
    # python make_golden.py [name ...]   (default: every fixture)
    for name in sys.argv[1:] or list(FIXTURES):
        FIXTURES[name]()
