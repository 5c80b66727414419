"""Failure detection on the GPU without a fault: a bounded device wait that
nothing ends gives up, reports its code through device memory, and the CUDA
context keeps working (the same wait guards every mbarrier of the tensor-core
kernels)."""

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives():
    from magic_b200 import Plan, _lib

    L = _lib.lib()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(L.mt_selftest_wait_timeout(C.c_void_p(status.data_ptr()), 1 << 12,
                                          C.c_void_p(stream)))
    torch.cuda.synchronize()
    assert status.item() == 99
    # the context is still usable: a split-precision round trip right after
    p = Plan(16, 1, precision="split")
    c = torch.zeros(p.lm_max, 2, dtype=torch.complex128, device="cuda")
    c[1:, :] = 1e-3
    c[torch.as_tensor(p.lm2m == 0)] = c[torch.as_tensor(p.lm2m == 0)].real.to(c.dtype)
    back = p.scal_to_SH(p.scal_to_spat(c))
    torch.cuda.synchronize()
    assert (back - c).abs().max().item() < 1e-7


def test_selftest_rejects_bad_arguments():
    from magic_b200 import _lib

    L = _lib.lib()
    assert L.mt_selftest_wait_timeout(None, 16, None) != 0
