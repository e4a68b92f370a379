"""Direct parity with the reference library: this library's results on the
inputs of tests/golden/ref_*.npz against the outputs the reference's own
tc_* routines produced on a B200 (make_golden.py). Both sides are FP16-operand
/ FP32-accumulate methods, so they agree to FP32-accumulation level; the FP64
SYRK is compared at FP64 level."""
import ctypes
import json
import os
import sys

import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)
import golden_inputs as gi  # noqa: E402


def load(name):
    z = np.load(os.path.join(GOLD, f"ref_{name}.npz"))
    return z, json.loads(str(z["meta"]))


def cm(x):
    """Device tensor whose storage is the column-major copy of x."""
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x).T)).cuda()


def host(t, rows, cols):
    return t.cpu().numpy().reshape(cols, rows).T


@pytest.mark.parametrize("name", ["syrk_small", "syrk_beta"])
def test_syrk_vs_reference(tblas, name):
    z, meta = load(name)
    n, k = meta["n"], meta["k"]
    A = gi.uniform(meta["seed"], (n, k))
    C0 = gi.uniform(meta["seed"] + 1, (n, n)) if meta["beta"] != 0 else np.zeros((n, n), np.float32)
    dC = cm(C0)
    tblas.ssyrk(cm(A), dC, n, k, n, n, meta["alpha"], meta["beta"], "N", meta["nb"])
    tblas.synchronize()
    got = host(dC, n, n)
    low = np.tril(np.ones((n, n), dtype=bool))
    _, err = orc.rel_errors(got, z["C"], low)
    assert err <= 2 * (1e-6 + 1e-8 * k), err


def test_syrk_vs_reference_recursive_path(tblas):
    z, meta = load("syrk_p2")
    n, k = meta["n"], meta["k"]
    A = gi.uniform(meta["seed"], (n, k))
    dC = torch.zeros(n * n, device="cuda")
    tblas.ssyrk(cm(A), dC, n, k, n, n, 1.0, 0.0, "N", meta["nb"])
    tblas.synchronize()
    got = host(dC, n, n)
    r, c = z["rows"], z["cols"]
    h = orc.h(A)
    scale = np.einsum("ij,ij->i", np.abs(h[r]), np.abs(h[c]))
    assert np.all(np.abs(got[r, c] - z["vals"]) <= 2 * (2e-6 + 2e-8 * k) * scale + 1e-30)


@pytest.mark.parametrize("name", ["trsm_p2", "trsm_small", "trsm_p2_nb512"])
def test_trsm_vs_reference(tblas, name):
    z, meta = load(name)
    m, n, nb = meta["m"], meta["n"], meta["nb"]
    A = gi.lower_tri(meta["seed"], n)
    B = gi.uniform(meta["seed"] + 1, (m, n))
    dB = cm(B)
    tblas.strsm("R", cm(A), dB, m, n, n, m, nb)
    tblas.synchronize()
    got = host(dB, m, n)
    _, err = orc.rel_errors(got, z["X"])
    exact = np.linalg.solve(A.astype(np.float64), B.astype(np.float64).T).T
    _, err_ref = orc.rel_errors(z["X"], exact)
    print(f"{name}: ours vs reference {err:.3e}; reference vs FP64 {err_ref:.3e}")
    assert err <= 3e-5


def test_syr2k_vs_reference(tblas):
    z, meta = load("syr2k_small")
    n, k = meta["n"], meta["k"]
    A = gi.uniform(meta["seed"], (n, k))
    B = gi.uniform(meta["seed"] + 1, (n, k))
    got = tblas.syr2k(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()).cpu().numpy()
    low = np.tril(np.ones((n, n), dtype=bool))
    _, err = orc.rel_errors(got, z["C"], low)
    assert err <= 2 * (1e-6 + 2e-8 * k), err


@pytest.mark.parametrize("name", ["trmm_small", "trmm_p2"])
def test_trmm_vs_reference(tblas, name):
    z, meta = load(name)
    m, n = meta["m"], meta["n"]
    A = np.tril(gi.uniform(meta["seed"], (m, m)))
    B = gi.uniform(meta["seed"] + 1, (m, n))
    got = tblas.trmm(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), 1.0, "L").cpu().numpy()
    _, err = orc.rel_errors(got, z["C"])
    assert err <= 2 * (1e-6 + 1e-8 * m), err


def test_symm_vs_reference(tblas):
    z, meta = load("symm_small")
    m = meta["m"]
    A = gi.uniform(meta["seed"], (m, m))
    B = gi.uniform(meta["seed"] + 1, (m, m))
    got = tblas.symm(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), 1.0, 0.0, None, "L").cpu().numpy()
    _, err = orc.rel_errors(got, z["C"])
    assert err <= 2 * (1e-6 + 1e-8 * m), err


def test_dsyrk_ozaki_vs_reference_fp64(tblas):
    z, meta = load("dsyrk_small")
    n, k = meta["n"], meta["k"]
    g = gi.rng(meta["seed"])
    A = g.standard_normal((n, k)) * np.exp(meta["phi"] * g.standard_normal((n, k)))
    lib = tblas.lib
    P, L = ctypes.c_void_p, ctypes.c_long
    lib.tb_dsyrk_ozaki.argtypes = [ctypes.c_char, ctypes.c_char, L, L, ctypes.c_double, P, L, ctypes.c_double, P, L,
                                   ctypes.c_int]
    dA = cm(A)
    dC = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    tblas._check(lib.tb_dsyrk_ozaki(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, 10))
    tblas.synchronize()
    got = host(dC, n, n)
    low = np.tril(np.ones((n, n), dtype=bool))
    _, err = orc.rel_errors(got, z["C"], low)
    assert err <= 1e-14, err
