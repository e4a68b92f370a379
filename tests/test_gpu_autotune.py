"""nb = TB_NB_AUTO on the GPU: the first call tunes (one cache entry per
key, nb from the candidate set), later calls reuse the entry, and the
results are those of the routine run with explicit parameters (checked
against the oracle model / the FP64 solution like the routine tests)."""
import numpy as np
import pytest
import torch

import tb_oracle as orc
import TensorBLAS as TB

pytestmark = pytest.mark.gpu


@pytest.fixture()
def fresh():
    TB.autotune_set_file(None)
    TB.lib.tb_autotune_clear()
    yield
    TB.lib.tb_autotune_clear()


def test_ssyrk_auto(fresh):
    g = np.random.Generator(np.random.PCG64(41))
    n, k = 1024, 768
    A = g.uniform(-1, 1, (n, k)).astype(np.float32)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()  # column-major n x k
    for rep in range(2):
        dC = torch.zeros(n * n, device="cuda")
        TB.ssyrk(dA, dC, n, k, n, n, 1.0, 0.0, "N", TB.NB_AUTO, TB.SPLIT)
        TB.synchronize()
        assert TB.autotune_entries() == 1
    choice = TB.autotune_get("ssyrk", "LN", n, k, TB.SPLIT)
    assert choice is not None and choice[1] in (0, 1)  # split precision: no narrow-engine candidate
    got = dC.cpu().numpy().reshape(n, n).T.astype(np.float64)
    exact = A.astype(np.float64) @ A.astype(np.float64).T
    low = np.tril(np.ones((n, n), dtype=bool))
    err = np.linalg.norm((got - exact)[low]) / np.linalg.norm(exact[low])
    assert err <= 2e-6


def test_strsm_auto(fresh):
    g = np.random.Generator(np.random.PCG64(43))
    m, n = 2048, 512
    A = (np.tril(g.uniform(-1, 1, (m, m)) / np.sqrt(m), -1) + np.diag(g.uniform(1, 2, m))).astype(np.float32)
    B = g.uniform(-1, 1, (m, n)).astype(np.float32)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    TB.strsm("L", dA, dB, m, n, m, m, TB.NB_AUTO, TB.SPLIT)
    TB.synchronize()
    nb, engine = TB.autotune_get("strsm", "L", m, n, TB.SPLIT)
    assert nb in (128, 256, 512) and engine in (0, 1)
    X = dB.cpu().numpy().T.astype(np.float64)
    exact = np.linalg.solve(A.astype(np.float64), B.astype(np.float64))
    _, err = orc.rel_errors(X, exact)
    assert err <= 2e-6
    # the same call again reuses the entry and gives the same result as the
    # explicit (nb, engine) it chose
    dB2 = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    TB.strsm("L", dA, dB2, m, n, m, m, TB.NB_AUTO, TB.SPLIT)
    TB.synchronize()
    assert TB.autotune_entries() == 1
    assert torch.equal(dB, dB2)


@pytest.mark.parametrize("uplo", ["L", "U"])
def test_ssyrk_splitk_wins_small_n_long_k(fresh, uplo):
    """n = 768, k = 16384 plain: the one-pass triangle has 12 tiles of
    128 x 256 for 148 SMs, so a split-K candidate (parts of K in one grouped
    launch plus a reduction) must beat both one-pass engines. The chosen form
    is checked against FP64 of the FP16-rounded operands, the other triangle
    stays untouched, and a second auto call reuses the entry and gives the
    same bits."""
    g = np.random.Generator(np.random.PCG64(47))
    n, k = 768, 16384
    A = g.uniform(-1, 1, (n, k)).astype(np.float32)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    C0 = g.uniform(-1, 1, (n, n)).astype(np.float32)
    dC = torch.from_numpy(np.ascontiguousarray(C0.T)).cuda().reshape(-1)
    TB._bind_stream(dA)
    TB._check(TB.lib.tb_ssyrk(uplo.encode(), b"N", n, k, 0.5, dA.data_ptr(), n, 2.0, dC.data_ptr(), n, TB.NB_AUTO,
                              TB.PLAIN))
    TB.synchronize()
    nb, engine, sk = TB.autotune_get_ex("ssyrk", uplo + "N", n, k, TB.PLAIN)
    assert sk > 1, "a split-K candidate should win at n = 768, k = 16384"
    got = dC.cpu().numpy().reshape(n, n).T.astype(np.float64)
    Ah = A.astype(np.float16).astype(np.float64)  # plain: FP16-rounded operands
    exact = 0.5 * (Ah @ Ah.T) + 2.0 * C0.astype(np.float64)
    tri = np.tril(np.ones((n, n), dtype=bool)) if uplo == "L" else np.triu(np.ones((n, n), dtype=bool))
    err = np.linalg.norm((got - exact)[tri]) / np.linalg.norm(exact[tri])
    assert err <= 1e-6 + 1e-8 * k
    assert np.array_equal(got[~tri], C0.astype(np.float64)[~tri])  # the other triangle is untouched
    # a second auto call reuses the entry and gives the same bits
    dC2 = torch.from_numpy(np.ascontiguousarray(C0.T)).cuda().reshape(-1)
    TB._check(TB.lib.tb_ssyrk(uplo.encode(), b"N", n, k, 0.5, dA.data_ptr(), n, 2.0, dC2.data_ptr(), n, TB.NB_AUTO,
                              TB.PLAIN))
    TB.synchronize()
    assert torch.equal(dC, dC2)


@pytest.mark.parametrize("uplo,n,k,parts", [("L", 500, 3000, 5), ("U", 333, 1100, 3), ("L", 1024, 4096, 16)])
def test_ssyrk_splitk_forced_entry(fresh, uplo, n, k, parts):
    """A cached split-K entry (put through tb_autotune_put_ex) drives the
    NB_AUTO call: ragged n and k, K parts of unequal length, beta = 0."""
    g = np.random.Generator(np.random.PCG64(53 + n))
    A = g.uniform(-1, 1, (n, k)).astype(np.float32)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    TB._check(TB.lib.tb_autotune_put_ex(b"ssyrk", (uplo + "N").encode(), n, k, TB.PLAIN, 256, 0, parts, 0.0))
    dC = torch.full((n * n,), 7.0, device="cuda")
    TB._bind_stream(dA)
    TB._check(TB.lib.tb_ssyrk(uplo.encode(), b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, TB.NB_AUTO,
                              TB.PLAIN))
    TB.synchronize()
    got = dC.cpu().numpy().reshape(n, n).T.astype(np.float64)
    Ah = A.astype(np.float16).astype(np.float64)
    exact = Ah @ Ah.T
    tri = np.tril(np.ones((n, n), dtype=bool)) if uplo == "L" else np.triu(np.ones((n, n), dtype=bool))
    err = np.linalg.norm((got - exact)[tri]) / np.linalg.norm(exact[tri])
    assert err <= 1e-6 + 1e-8 * k
    assert np.all(got[~tri] == 7.0)


def _run_auto(routine, dA, dB, n1, n2):
    """One NB_AUTO call of tb_ssyr2k ('L', 'N': n = n1, k = n2) or tb_strmm
    ('U': m = n1, n = n2) in plain precision on fresh zero outputs."""
    size = n1 * n1 if routine == "ssyr2k" else n1 * n2
    dC = torch.zeros(size, device="cuda")
    TB._bind_stream(dA)
    if routine == "ssyr2k":
        TB._check(TB.lib.tb_ssyr2k(b"L", b"N", n1, n2, 1.0, dA.data_ptr(), n1, dB.data_ptr(), n1, 0.0, dC.data_ptr(),
                                   n1, TB.NB_AUTO, TB.PLAIN))
    else:
        TB._check(TB.lib.tb_strmm(b"U", n1, n2, 1.0, dA.data_ptr(), n1, dB.data_ptr(), n1, dC.data_ptr(), n1,
                                  TB.NB_AUTO, TB.PLAIN))
    TB.synchronize()
    return dC


@pytest.mark.parametrize("routine,n1,n2", [("ssyr2k", 1024, 8192), ("strmm", 4096, 256), ("ssyr2k", 1000, 3000)])
def test_engines_give_the_same_bits_and_tuner_picks_one(fresh, routine, n1, n2):
    """Plain long-K launches on CTA pairs (engine 1, 256 x 256), single-CTA
    128 x 256 tiles (0) or single-CTA 128 x 128 tiles (2, the narrow engine,
    twice the tiles of 0 where the wider tiles leave SMs idle): each element
    is the same K-ordered FP32 sum of the same FP16 products, so a cached
    entry naming any of them gives the same bits; the tuner's own choice is
    one of the three and gives those bits too; the result matches FP64 of
    the FP16-rounded operands."""
    g = np.random.Generator(np.random.PCG64(59 + n1))
    if routine == "ssyr2k":
        n, k = n1, n2
        A = g.uniform(-1, 1, (n, k)).astype(np.float32)
        B = g.uniform(-1, 1, (n, k)).astype(np.float32)
        flags = "LN"
    else:
        m, n = n1, n2
        A = np.triu(g.uniform(-1, 1, (m, m))).astype(np.float32)
        B = g.uniform(-1, 1, (m, n)).astype(np.float32)
        flags = "U"
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    outs = {}
    for e in (0, 1, 2):
        TB.lib.tb_autotune_clear()
        TB._check(TB.lib.tb_autotune_put(routine.encode(), flags.encode(), n1, n2, TB.PLAIN, 256, e, 0.0))
        outs[e] = _run_auto(routine, dA, dB, n1, n2)
    assert torch.equal(outs[0], outs[2]) and torch.equal(outs[1], outs[2])
    TB.lib.tb_autotune_clear()
    tuned = _run_auto(routine, dA, dB, n1, n2)
    nb, engine = TB.autotune_get(routine, flags, n1, n2, TB.PLAIN)
    assert engine in (0, 1, 2)
    assert torch.equal(tuned, outs[2])
    Ah = A.astype(np.float16).astype(np.float64)
    Bh = B.astype(np.float16).astype(np.float64)
    if routine == "ssyr2k":
        got = tuned.cpu().numpy().reshape(n1, n1).T.astype(np.float64)
        exact = Ah @ Bh.T + Bh @ Ah.T
        sel = np.tril(np.ones((n1, n1), dtype=bool))
        K = 2 * n2
    else:
        got = tuned.cpu().numpy().reshape(n2, n1).T.astype(np.float64)
        exact = Ah @ Bh
        sel = np.ones_like(exact, dtype=bool)
        K = n1
    err = np.linalg.norm((got - exact)[sel]) / np.linalg.norm(exact[sel])
    assert err <= 1e-6 + 1e-8 * K

