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


def test_device_status_surfaces_through_the_plan():
    """A split call's workspace reads 0 after a good call.  A code planted in the
    status word by the self-test wait (a bounded wait nothing ends) is returned
    by mt_device_status and raised by the plan's watch, and the plan keeps
    working once the workspace is cleared by the next call."""
    from magic_b200 import MagicError, Plan, _lib

    L = _lib.lib()
    p = Plan(16, 1, precision="split")
    c = torch.zeros(p.lm_max, 2, dtype=torch.complex128, device="cuda")
    c[1:, :] = 1e-3
    c[torch.as_tensor(p.lm2m == 0)] = c[torch.as_tensor(p.lm2m == 0)].real.to(c.dtype)
    ws = torch.zeros(L.mt_transform_workspace(p._h, 2, 1), dtype=torch.uint8, device="cuda")
    g = torch.empty(2, p.n_theta_max, p.n_phi_max, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.mt_scal_to_spat(p._h, C.c_void_p(c.data_ptr()), 2, 2, C.c_void_p(g.data_ptr()),
                                 C.c_void_p(ws.data_ptr()), ws.numel(), stream))
    assert p.device_status(ws) == 0
    _lib.check(L.mt_selftest_wait_timeout(C.c_void_p(ws.data_ptr()), 1 << 12, stream))
    assert p.device_status(ws) == 99
    p._watch(ws, "planted")
    with pytest.raises(MagicError, match="code 99"):
        p.poll_status(block=True)
    back = p.scal_to_SH(p.scal_to_spat(c))
    p.poll_status(block=True)
    assert (back - c).abs().max().item() < 1e-7


def test_noalloc_status_reads_zero_after_a_good_call():
    from magic_b200 import Plan, _lib

    L = _lib.lib()
    p = Plan(16, 1, precision="split")
    c = torch.zeros(p.lm_max, 1, dtype=torch.complex128, device="cuda")
    c[1:, :] = 1e-3
    g = torch.empty(1, p.n_theta_max, p.n_phi_max, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.mt_scal_to_spat_noalloc(p._h, C.c_void_p(c.data_ptr()), 1, 1,
                                         C.c_void_p(g.data_ptr()), stream))
    code = C.c_int(-1)
    _lib.check(L.mt_noalloc_status(C.byref(code), stream))
    assert code.value == 0
    ref = p.scal_to_spat(c)
    torch.cuda.synchronize()
    assert (g - ref).abs().max().item() <= 1e-7 * ref.abs().max().item()
