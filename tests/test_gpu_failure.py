"""Failure path of the bounded device waits, exercised without a GPU fault.

tb_debug_stall(tile, wait_ns) makes the GEMM producers skip the operand
loads of one tile, so the MMA issuer's wait for them can never be satisfied,
and shortens every bounded device wait to `wait_ns`. The kernel then records
a timeout in the device error block, lets its own copies and MMAs retire,
frees its TMEM and returns: tb_synchronize reports TB_ERROR_TIMEOUT, the
reference-facing wrappers return 1, and the context stays usable (the next
call, with the hook off, gives the right answer). Each case covers one
engine: CTA-pair tiles (plain, n >= 512), single-CTA tiles (split), the
prefetch variant (short K) and a grouped launch with the device-side tile
scheduler (a batch).
"""
import numpy as np
import pytest
import torch

import tb_oracle as orc

pytestmark = pytest.mark.gpu

TIMEOUT = 4  # TB_ERROR_TIMEOUT
LIMIT_NS = 20_000_000  # 20 ms: every wait of the stalled launch gives up after this


@pytest.fixture()
def stall(tblas):
    """Turns the hook on for tile 0 and always turns it off again."""
    tblas._check(tblas.lib.tb_debug_stall(0, LIMIT_NS))
    try:
        yield
    finally:
        tblas.lib.tb_debug_stall(-1, 0)
        tblas.lib.tb_synchronize()  # clears a code a failed assertion may have left


def _syrk_inputs(n, k, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    A = g.uniform(-1, 1, (n, k)).astype(np.float32)
    return A, torch.from_numpy(np.ascontiguousarray(A.T)).cuda()


def _check_syrk(tblas, A, dA, n, k, precision):
    dC = torch.zeros(n, n, device="cuda")
    tblas._bind_stream(dA)
    tblas._check(tblas.lib.tb_ssyrk(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, 256, precision))
    tblas.synchronize()
    low = np.tril(np.ones((n, n), dtype=bool))
    _, err = orc.rel_errors(dC.cpu().numpy().T, orc.syrk_model(A, split=bool(precision)), low)
    assert err <= (2e-6 if precision else 1e-6 + 1e-8 * k)


@pytest.mark.parametrize("precision,n,k", [(0, 512, 2048),   # CTA-pair engine
                                           (1, 384, 2048),   # single-CTA split tiles
                                           (1, 384, 200)])   # prefetch (short-K) variant
def test_stalled_tile_reports_timeout_and_context_recovers(tblas, precision, n, k):
    A, dA = _syrk_inputs(n, k, 31 + n)
    dC = torch.zeros(n, n, device="cuda")
    tblas._bind_stream(dA)
    tblas._check(tblas.lib.tb_debug_stall(0, LIMIT_NS))
    try:
        st = tblas.lib.tb_ssyrk(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0, dC.data_ptr(), n, 256, precision)
        assert st == 0  # queued; the wait runs out on the device
        assert tblas.lib.tb_synchronize() == TIMEOUT
        assert b"timed out" in tblas.lib.tb_last_error()
    finally:
        tblas.lib.tb_debug_stall(-1, 0)
    assert tblas.lib.tb_synchronize() == 0  # the code was read and cleared
    _check_syrk(tblas, A, dA, n, k, precision)


def test_wrapper_returns_error_on_timeout(tblas, stall):
    n, k = 512, 1024
    dA = torch.rand(n, k, device="cuda") * 2 - 1  # row-major n x k, as the reference's wrapper takes it
    dC = torch.zeros(n, n, device="cuda")
    tblas._bind_stream(dA)
    assert tblas.lib.tc_syrk_wrapper(n, k, dA.data_ptr(), dC.data_ptr(), 256) == 1
    tblas.lib.tb_debug_stall(-1, 0)
    assert tblas.lib.tc_syrk_wrapper(n, k, dA.data_ptr(), dC.data_ptr(), 256) == 0
    ref = dA.double() @ dA.double().T
    assert float((dC.double() - ref).norm() / ref.norm()) < 1e-3


def test_grouped_launch_reports_timeout(tblas, stall):
    sizes = [200, 320, 256, 96]
    kinds, As, BC = [], [], []
    for i, m in enumerate(sizes):
        kinds.append(i % 2)
        if i % 2 == 0:
            As.append(torch.rand(m, m, device="cuda") * 2 - 1)
            BC.append(torch.zeros(m, m, device="cuda"))
        else:
            lt = torch.tril(torch.rand(m, m, device="cuda") * 2 - 1, -1) / m ** 0.5
            As.append((lt + torch.diag(torch.rand(m, device="cuda") + 1)).t().contiguous())
            BC.append(torch.rand(m, m, device="cuda") * 2 - 1)
    B0 = [b.clone() for b in BC]
    batch = tblas.Batch(kinds, As, BC, precision=tblas.SPLIT)
    try:
        batch.run()
        assert tblas.lib.tb_synchronize() == TIMEOUT
        tblas.lib.tb_debug_stall(-1, 0)
        for b, b0 in zip(BC, B0):
            b.copy_(b0)
        batch.run()
        tblas.synchronize()
    finally:
        batch.close()
    a, c = As[0].cpu().double().T, BC[0].cpu().double().T  # logical A, C (column-major storage)
    ref = a @ a.T
    low = torch.tril(torch.ones_like(ref, dtype=torch.bool))
    assert float((c - ref)[low].norm() / ref[low].norm()) < 2e-6
