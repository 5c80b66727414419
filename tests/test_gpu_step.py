"""A whole CNAB2 time step of the Boussinesq MHD dynamo on the GPU
(magic_b200.step.BoussinesqStep: fused nonlinear stage, explicit terms,
implicit solves S, Z, W, B), checked as a composition of the entry points
that the other GPU tests pin against the reference: repeated steps stay
finite and reproduce bit for bit, the split-precision and FP64 stages agree
to the split tolerance after a few steps, and without buoyancy or rotation
the kinetic and magnetic parts of a small perturbation only decay."""

import pytest
import torch

pytestmark = pytest.mark.gpu


def _energy(st):
    return sum(float((st.f[k].abs() ** 2).sum()) for k in ("w", "z", "b", "aj"))


def _run(precision, n, **kw):
    from magic_b200.step import BoussinesqStep

    st = BoussinesqStep(32, 33, precision=precision, **kw)
    st.init_random(seed=1, amp=1e-3)
    dts = []
    for _ in range(n):
        dts.append(st.step())
    torch.cuda.synchronize()
    return st, dts


def test_step_is_finite_and_deterministic():
    a, dts = _run("fp64", 3)
    b, _ = _run("fp64", 3)
    for k in a.f:
        assert torch.isfinite(torch.view_as_real(a.f[k])).all(), k
        assert torch.equal(a.f[k], b.f[k]), k
    assert all(torch.isfinite(d).all() for pair in dts for d in pair)


def test_split_stage_tracks_fp64_stage():
    a, _ = _run("fp64", 3)
    b, _ = _run("split", 3)
    for k in ("w", "z", "s", "b", "aj"):
        e = ((a.f[k] - b.f[k]).abs().max() / a.f[k].abs().max()).item()
        assert e < 1e-4, (k, e)


def test_pure_diffusion_decays():
    a, _ = _run("fp64", 1, ra=0.0, ek=1e6)
    e0 = _energy(a)
    for _ in range(5):
        a.step()
    torch.cuda.synchronize()
    assert _energy(a) < e0
