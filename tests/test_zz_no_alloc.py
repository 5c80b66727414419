"""The allocation-free scalar synthesis (mt_scal_to_spat_noalloc).

Some callers cannot allocate device memory while they run: a host code that
links this library through its C ABI and budgets all GPU memory once at
start-up, or a process whose device memory is owned by another allocator.
For them the library offers one entry point whose workspace is a fixed
16 MiB array inside the library.  These tests call it through the C ABI and
check it against the workspace-taking mt_scal_to_spat (1e-12 relative, the
FP64 tolerance of the other tests) on two calls in a row, the second with
different data so leftovers of the first call would show, and check that an
oversized batch is refused before any launch.  Split-precision plans keep
their operand images in the same array, so their limit is lower (the
workspace query gives it); their device status is read with
mt_noalloc_status.  This file is collected last so a failure here comes after
every other test has run.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _spec(plan, B, seed):
    rng = np.random.default_rng(seed)
    amp = (plan.lm2l + 1.0) ** -1.5
    x = (rng.standard_normal((plan.lm_max, B)) + 1j * rng.standard_normal((plan.lm_max, B)))
    return torch.as_tensor(x * amp[:, None]).cuda()


def _noalloc(plan, Slm):
    from magic_b200 import _lib

    B = Slm.shape[1]
    out = torch.empty(B, plan.n_theta_max, plan.n_phi_max, dtype=torch.float64, device="cuda")
    rc = _lib.lib().mt_scal_to_spat_noalloc(
        plan._h, ctypes.c_void_p(Slm.data_ptr()), Slm.stride(0), B,
        ctypes.c_void_p(out.data_ptr()),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc)
    return out


def test_noalloc_matches_workspace_entry_point_twice():
    from magic_b200 import Plan

    plan = Plan(63)
    for seed, B in ((1, 5), (2, 7)):
        Slm = _spec(plan, B, seed)
        ref = plan.scal_to_spat(Slm)
        got = _noalloc(plan, Slm)
        torch.cuda.synchronize()
        err = (got - ref).abs().max().item() / ref.abs().max().item()
        assert err < 1e-12, err


def test_noalloc_refuses_oversized_batch():
    from magic_b200 import Plan, _lib

    plan = Plan(63)
    per_col = plan.n_m_max * plan.n_theta_max * 16
    B = (16 << 20) // per_col + 1
    Slm = _spec(plan, B, 3)
    out = torch.empty(B, plan.n_theta_max, plan.n_phi_max, dtype=torch.float64, device="cuda")
    L = _lib.lib()
    rc = L.mt_scal_to_spat_noalloc(plan._h, ctypes.c_void_p(Slm.data_ptr()), Slm.stride(0), B,
                                   ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 4  # MT_ERR_WORKSPACE
    assert b"16 MiB" in L.mt_last_error()


def test_noalloc_split_plan_matches_and_reports_status():
    """A split-precision plan keeps its operand images in the same fixed array;
    the allocation-free call gives the same grids as the workspace-taking call
    (same kernels, so to FP64 rounding of the same arithmetic), and its device
    status, which only mt_noalloc_status can read, is 0."""
    from magic_b200 import Plan, _lib

    plan = Plan(63, precision="split")
    L = _lib.lib()
    for seed, B in ((4, 2), (5, 3)):
        assert L.mt_transform_workspace(plan._h, B, 1) <= 16 << 20
        Slm = _spec(plan, B, seed)
        ref = plan.scal_to_spat(Slm)
        got = _noalloc(plan, Slm)
        code = ctypes.c_int(-1)
        _lib.check(L.mt_noalloc_status(ctypes.byref(code),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        assert code.value == 0
        err = (got - ref).abs().max().item() / ref.abs().max().item()
        assert err < 1e-12, err


def test_noalloc_split_plan_refuses_oversized_batch():
    from magic_b200 import Plan, _lib

    plan = Plan(63, precision="split")
    L = _lib.lib()
    B = 1
    while L.mt_transform_workspace(plan._h, B, 1) <= 16 << 20:
        B += 1
    Slm = _spec(plan, B, 6)
    out = torch.empty(B, plan.n_theta_max, plan.n_phi_max, dtype=torch.float64, device="cuda")
    rc = L.mt_scal_to_spat_noalloc(plan._h, ctypes.c_void_p(Slm.data_ptr()), Slm.stride(0), B,
                                   ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 4  # MT_ERR_WORKSPACE
    assert b"16 MiB" in L.mt_last_error()
