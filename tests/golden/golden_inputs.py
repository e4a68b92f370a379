"""Seeded inputs shared by the golden-vector generator and the tests.

Every fixture in this directory stores only the seed and shape of its
inputs; both the generator (run once against the reference library) and the
tests rebuild the same FP32 column-major matrices from NumPy's PCG64.
"""
import numpy as np


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def uniform(seed, shape, lo=-1.0, hi=1.0):
    return rng(seed).uniform(lo, hi, shape).astype(np.float32)


def lower_tri(seed, n):
    """Lower-triangular A with off-diagonal U[-1,1]/sqrt(n), diagonal U[1,2]; zero upper."""
    g = rng(seed)
    A = np.tril(g.uniform(-1, 1, (n, n)) / np.sqrt(n), -1) + np.diag(g.uniform(1, 2, n))
    return A.astype(np.float32)


def wide_range(seed, shape):
    """N(0,1) * 2^U(-8,8), exponent drawn per element (SYR2K/TRMM/SYMM configs)."""
    g = rng(seed)
    return (g.standard_normal(shape) * np.exp2(g.uniform(-8, 8, shape))).astype(np.float32)


def checksum(x):
    x = np.ascontiguousarray(x)
    return float(np.sum(x.astype(np.float64) * (1.0 + np.arange(x.size, dtype=np.float64).reshape(x.shape) % 7)))
