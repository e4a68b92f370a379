"""Batched uneven SYRK/TRSM instances (grouped launches) against the oracle
and against the per-instance entry points; the batch replayed from a CUDA
graph must give the same results."""
import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu


def _instances(seed, count, lo=64, hi=700):
    g = np.random.Generator(np.random.PCG64(seed))
    ns = np.round(np.exp(g.uniform(np.log(lo), np.log(hi), count))).astype(int)
    kinds, A, BC, host = [], [], [], []
    for i, n in enumerate(ns):
        kind = i % 2
        if kind == 0:
            a = g.uniform(-1, 1, (n, n)).astype(np.float32)
            bc = np.zeros((n, n), np.float32)
        else:
            a = (np.tril(g.uniform(-1, 1, (n, n)) / np.sqrt(n), -1) + np.diag(g.uniform(1, 2, n))).astype(np.float32)
            bc = g.uniform(-1, 1, (n, n)).astype(np.float32)
        kinds.append(kind)
        A.append(torch.from_numpy(np.ascontiguousarray(a.T)).cuda())
        BC.append(torch.from_numpy(np.ascontiguousarray(bc.T)).cuda())
        host.append((a, bc))
    return kinds, A, BC, host


def _check_results(kinds, BC, host, precision):
    worst = 0.0
    for kind, bc, (a, b0) in zip(kinds, BC, host):
        n = a.shape[0]
        got = bc.cpu().numpy().T
        if kind == 0:
            model = orc.syrk_model(a, split=bool(precision))
            low = np.tril(np.ones((n, n), dtype=bool))
            _, err = orc.rel_errors(got, model, low)
            tol = 2e-6 if precision else 1e-6 + 1e-8 * n
        else:
            # orders below 2048 are FP32-accurate in both precisions
            exact = np.linalg.solve(a.astype(np.float64), b0.astype(np.float64).T).T
            _, err = orc.rel_errors(got, exact)
            tol = 2e-6
        worst = max(worst, err / tol)
        assert err <= tol, (kind, n, err)
    return worst


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_oracle(tblas, precision):
    kinds, A, BC, host = _instances(3 + precision, 24)
    batch = tblas.Batch(kinds, A, BC, precision=precision)
    batch.run()
    tblas.synchronize()
    _check_results(kinds, BC, host, precision)
    batch.close()


def test_batch_cuda_graph_replay(tblas):
    kinds, A, BC, host = _instances(9, 16)
    B0 = [b.clone() for b in BC]
    batch = tblas.Batch(kinds, A, BC, precision=tblas.SPLIT)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        batch.run()  # warm-up outside capture
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        batch.run()
    for rep in range(2):
        for b, b0 in zip(BC, B0):
            b.copy_(b0)
        graph.replay()
        torch.cuda.synchronize()
        _check_results(kinds, BC, host, 1)
    del graph
    batch.close()
