"""Argument checks of the Python front-end, on the CPU.

A tensor of the wrong shape, dtype or device would make the kernels read or
write outside it (or hand a host pointer to the GPU), so the front-end
rejects it before any device work: ValueError for a shape, TypeError for a
dtype or device. With CPU tensors of the right shapes every call must stop
at the device check, which shows that no check runs after a library call.
"""
import pytest
import torch

import TensorBLAS as TB


def cpu(*shape, dtype=torch.float32):
    return torch.zeros(*shape, dtype=dtype)


@pytest.mark.parametrize("call", [
    lambda: TB.syrk(cpu(8)),                                    # A not 2-D
    lambda: TB.syrk(cpu(8, 4), C=cpu(8, 9)),                    # C not n x n
    lambda: TB.syr2k(cpu(8, 4), cpu(8, 5)),                     # B not n x k
    lambda: TB.syr2k(cpu(8, 4), cpu(8, 4), C=cpu(4, 4)),        # C not n x n
    lambda: TB.trsm(cpu(6, 6), cpu(8, 3), side="L"),            # A not m x m
    lambda: TB.trsm(cpu(8, 8), cpu(8, 3), side="R"),            # A not n x n
    lambda: TB.trsm(cpu(8, 7), cpu(8, 3), side="L"),            # A not square
    lambda: TB.trmm(cpu(5, 5), cpu(8, 3)),                      # A not m x m
    lambda: TB.symm(cpu(8, 8), cpu(8, 3), C=cpu(3, 8)),         # C not m x n
    lambda: TB.symm(cpu(8, 7), cpu(8, 3)),                      # A not m x m
    lambda: TB.tc_syrk(cpu(2, 3, 4)),                           # A not 2-D
    lambda: TB.tc_trsm(cpu(6, 5), cpu(4, 6)),                   # A not square
    lambda: TB.tc_trsm(cpu(6, 6), cpu(4, 5)),                   # B not m x n
    lambda: TB.Batch([0, 1], [cpu(4, 4), cpu(5, 5)], [cpu(4, 4)]),          # one BC missing
    lambda: TB.Batch([0, 2], [cpu(4, 4), cpu(5, 5)], [cpu(4, 4), cpu(5, 5)]),  # unknown kind
    lambda: TB.Batch([0], [cpu(4, 5)], [cpu(4, 5)]),                         # not square
    lambda: TB.Batch([1], [cpu(4, 4)], [cpu(5, 5)]),                         # BC of another size
])
def test_wrong_shapes_are_rejected(call):
    with pytest.raises(ValueError):
        call()


@pytest.mark.parametrize("call", [
    lambda: TB.syrk(cpu(8, 4)),
    lambda: TB.syrk(cpu(8, 4), C=cpu(8, 8)),
    lambda: TB.syr2k(cpu(8, 4), cpu(8, 4), C=cpu(8, 8)),
    lambda: TB.trsm(cpu(8, 8), cpu(8, 3), side="L"),
    lambda: TB.trsm(cpu(3, 3), cpu(8, 3), side="R"),
    lambda: TB.trmm(cpu(8, 8), cpu(8, 3)),
    lambda: TB.symm(cpu(8, 8), cpu(8, 3), C=cpu(8, 3)),
    lambda: TB.tc_syrk(cpu(8, 4)),
    lambda: TB.tc_trsm(cpu(6, 6), cpu(4, 6)),
    lambda: TB.ssyrk(cpu(32), cpu(64), 8, 4, 8, 8),
    lambda: TB.strsm("L", cpu(64), cpu(24), 8, 3, 8, 8),
    lambda: TB.sgemm("N", "N", 8, 8, 8, 1.0, cpu(64), 8, cpu(64), 8, 0.0, cpu(64), 8),
    lambda: TB.Batch([0, 1], [cpu(4, 4), cpu(25)], [cpu(4, 4), cpu(5, 5)]),
])
def test_host_tensors_are_rejected_before_device_work(call):
    with pytest.raises(TypeError, match="CUDA"):
        call()


def test_wrong_dtype_is_rejected():
    with pytest.raises(TypeError, match="float32"):
        TB.syrk(cpu(8, 4, dtype=torch.float64))
    with pytest.raises(TypeError, match="float32"):
        TB.ssyrk(cpu(32, dtype=torch.float16), cpu(64), 8, 4, 8, 8)
