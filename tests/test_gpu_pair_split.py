"""Long split-precision launches (hi/lo operands, three products, RN folds
every kchunk K-blocks) without FP16 side copies run on CTA pairs with
256 x 128 tiles; with TB_GEMM_PAIR_SPLIT=0 they run on single-CTA 128 x 128
tiles. Each output element sees the same three products per 16-deep K step,
in the same order, folded at the same K-block boundaries, so the split
results must be bit-identical under both settings: SYRK ('N' and 'T',
ragged n), SYR2K, lower TRMM, SYMM with beta != 0, SGEMM with both
transposes, and TRSM left and right. Upper TRMM is the exception: a pair
tile's K range is the union of its two 128-row halves' ranges, and in the
upper triangle those start at different K blocks, so the fold boundaries
of one half move (the extra products are of stored zeros); it is checked
against FP64 only, like every routine here. The switch is read once per
process, so each setting runs in its own subprocess."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import hashlib, sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
import TensorBLAS as TB
S = TB.SPLIT
g = np.random.Generator(np.random.PCG64(29))
digests = {}
errs = {}

def rnd(*shape):
    return torch.from_numpy(g.uniform(-1, 1, shape).astype(np.float32)).cuda()

def err(name, got, ref):
    ref = np.asarray(ref, dtype=np.float64)
    errs[name] = float(np.linalg.norm(np.asarray(got, dtype=np.float64) - ref) / np.linalg.norm(ref))

def take(name, t, ref):
    TB.synchronize()
    x = t.cpu().numpy()
    digests[name] = hashlib.sha1(x.tobytes()).hexdigest()
    err(name, x, ref)

for n, k in ((1536, 2048), (1300, 1100)):
    A = rnd(n, k)
    C = TB.syrk(A, precision=S)
    Ad = A.cpu().numpy().astype(np.float64)
    take(f"syrk{n}", torch.tril(C), np.tril(Ad @ Ad.T))
# 'T': C = A^T A for a k x n column-major A (a row-major n x k torch tensor)
n, k = 1280, 1536
At = rnd(n, k)
Ct = torch.zeros(n, n, device="cuda")
TB._bind_stream(At)
TB.ssyrk(At, Ct, n, k, k, n, 1.0, 0.0, "T", 256, S)
Ad = At.cpu().numpy().astype(np.float64)
take("syrkT", torch.triu(Ct), np.triu(Ad @ Ad.T))  # column-major C's lower = row-major's upper

n, k = 1024, 1536
A, B = rnd(n, k), rnd(n, k)
Ad, Bd = A.cpu().numpy().astype(np.float64), B.cpu().numpy().astype(np.float64)
take("syr2k", torch.tril(TB.syr2k(A, B, precision=S)), np.tril(Ad @ Bd.T + Bd @ Ad.T))

m, n = 1536, 1024
T = rnd(m, m)
Bm = rnd(m, n)
Td, Bd = T.cpu().numpy().astype(np.float64), Bm.cpu().numpy().astype(np.float64)
take("trmmL", TB.trmm(T, Bm, uplo="L", precision=S), np.tril(Td) @ Bd)
take("trmmU", TB.trmm(T, Bm, uplo="U", precision=S), np.triu(Td) @ Bd)

Sy = rnd(m, m)
C0 = rnd(m, n)
Sd = np.tril(Sy.cpu().numpy().astype(np.float64))
Sd = Sd + np.tril(Sd, -1).T
take("symm", TB.symm(Sy, Bm, alpha=1.0, beta=0.5, C=C0, precision=S), Sd @ Bd + 0.5 * C0.cpu().numpy())

for ta, tb in (("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")):
    mm, nn, kk = 1152, 1280, 1536
    Ag = rnd(kk, mm) if ta == "N" else rnd(mm, kk)  # column-major storage of op(A)'s source
    Bg = rnd(nn, kk) if tb == "N" else rnd(kk, nn)
    Cg = torch.zeros(nn, mm, device="cuda")
    TB._bind_stream(Ag)
    TB.sgemm(ta, tb, mm, nn, kk, 1.0, Ag, mm if ta == "N" else kk, Bg, kk if tb == "N" else nn, 0.0, Cg, mm, S)
    a = Ag.cpu().numpy().astype(np.float64).T
    b = Bg.cpu().numpy().astype(np.float64).T
    opa = a if ta == "N" else a.T
    opb = b if tb == "N" else b.T
    take(f"gemm{ta}{tb}", Cg, (opa @ opb).T)

for side, m, n in (("L", 4096, 1536), ("R", 1536, 4096)):
    nt = m if side == "L" else n
    L = (np.tril(g.uniform(-1, 1, (nt, nt)) / np.sqrt(nt), -1) + np.diag(g.uniform(1, 2, nt))).astype(np.float32)
    Bt = g.uniform(-1, 1, (m, n)).astype(np.float32)
    X = TB.trsm(torch.from_numpy(L).cuda(), torch.from_numpy(Bt).cuda(), side=side, nb=512, precision=S)
    Ld, Btd = L.astype(np.float64), Bt.astype(np.float64)
    ref = np.linalg.solve(Ld, Btd) if side == "L" else np.linalg.solve(Ld, Btd.T).T
    take(f"trsm{side}", X, ref)

print("ERRS", repr(errs))
print("DIGESTS", repr(digests))
"""


def _run(pair_split):
    env = dict(os.environ, TB_GEMM_PAIR_SPLIT=pair_split)
    out = subprocess.run([sys.executable, "-c", SCRIPT, os.path.join(ROOT, "tensor-blas_b200", "python")], env=env,
                         capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = out.stdout.strip().splitlines()
    errs = eval(lines[-2].split(" ", 1)[1])
    digests = eval(lines[-1].split(" ", 1)[1])
    return digests, errs


def test_split_pair_tiles_match_single_cta_bits_and_fp64():
    pair_digest, errs = _run("1")
    for name, e in errs.items():
        assert e < 2e-6, (name, e)
    single_digest, _ = _run("0")
    differ = sorted(k for k in pair_digest if pair_digest[k] != single_digest[k] and k != "trmmU")
    assert not differ, differ
