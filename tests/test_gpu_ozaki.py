"""GPU parity of the digit-split (ozaki) fused nonlinear stage: int8 digit planes
of the Legendre operands on the tcgen05 integer pipe with exact int32
accumulation (six digits, 21 digit pairs per K chunk), FP64 phi stage, against
the oracle's FP64 restatement of the radial loop.

Tolerance 5e-13 l_max^2 of each output's scale (the vector pair's
max(|S|, |T|) for the S/T outputs) and on the Courant steps.  The digits carry
41 significant bits relative to the largest value of each operand row, and in
the analysis a row runs over theta: the vector outputs' 1/sin^2(theta) weight
makes the rows near the poles the largest by ~n_theta^2, so the equatorial
values keep fewer bits.  Measured with these white-noise spectra (amplitude
(l+1)^-1.5): 4.9e-11 (l_max 16), 3.1e-10 (32), 8.7e-10 (63), 2.1e-9 (127),
1.3e-8 (255), 3.3e-8 (383), largest in Advt/Advp.  Whole runs stay within the
north star's bounds (tests/test_gpu_step.py).  The l_max = 255 case is the
benchmark's horizontal grid (n_theta 384, n_phi 768), l_max = 383 the largest
(n_phi 1152)."""

import numpy as np
import pytest
import torch

from oracle import grid as og
from oracle import stage as ostage

pytestmark = pytest.mark.gpu

CASES = [
    # l_max, minc, n_r, l_mag, l_chem
    (16, 1, 5, True, False),
    (32, 4, 7, True, True),
    (20, 1, 6, False, True),
    (16, 1, 4, False, False),
    (63, 1, 9, True, False),
    (127, 1, 4, True, False),
    (255, 1, 3, True, False),
    (383, 1, 3, False, False),
    # the other warp-FFT row lengths of the FP64 phi kernel (n_phi 256, 512, 1024)
    (85, 1, 3, True, False),
    (170, 1, 3, True, True),
    (341, 1, 3, False, False),
]
PAIR = {"Advt": "Advp", "Advp": "Advt", "VxBt": "VxBp", "VxBp": "VxBt"}


def _tol(l_max):
    return 5e-13 * l_max ** 2


def _fields(g, N, rng, l_mag, l_chem):
    amp = (g.lm2l + 1.0) ** -1.5

    def spec():
        x = (rng.standard_normal((g.lm_max, N)) + 1j * rng.standard_normal((g.lm_max, N)))
        x = x * amp[:, None]
        x[g.lm2m == 0] = x[g.lm2m == 0].real
        return x

    names = ["w", "dw", "ddw", "z", "dz", "s"] + (["b", "db", "ddb", "aj", "dj"] if l_mag else [])
    names += ["xi"] if l_chem else []
    return {k: spec() for k in names}


@pytest.mark.parametrize("l_max,minc,N,l_mag,l_chem", CASES)
def test_ozaki_stage_matches_oracle(l_max, minc, N, l_mag, l_chem):
    from magic_b200 import Plan

    g = og.Grid(l_max, minc)
    p = Plan(l_max, minc, precision="ozaki")
    rng = np.random.default_rng(7 * l_max + N)
    f = _fields(g, N, rng, l_mag, l_chem)
    prof = ostage.bouss_profiles(N, l_max=l_max)
    LF, cf, af, opm = 200.0, 2.5, 1.0, 0.2
    ref, rdt, rdh = ostage.nl_bouss_stage(g, f, prof, LF, cf, af, opm, l_mag, l_chem)
    cu = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()
    work = torch.zeros(p.nl_bouss_workspace(N, l_mag, l_chem), dtype=torch.uint8, device="cuda")
    out, dt, dh = p.nl_bouss({k: cu(v) for k, v in f.items()}, {k: cu(v) for k, v in prof.items()},
                             LF, cf, af, opm, l_mag=l_mag, l_chem=l_chem, work=work)
    torch.cuda.synchronize()
    assert p.device_status(work) == 0, "device wait timed out"
    assert set(out) == set(ref)
    worst = {}
    for k in ref:
        got = out[k].cpu().numpy()
        assert np.all(got[:, 0] == 0) and np.all(got[:, -1] == 0), k
        scale = np.abs(ref[k]).max()
        if k in PAIR:
            scale = max(scale, np.abs(ref[PAIR[k]]).max())
        worst[k] = np.abs(got - ref[k]).max() / scale
    print("ozaki stage errors", {k: f"{v:.1e}" for k, v in worst.items()})
    for k, v in worst.items():
        assert v < _tol(l_max), (k, v)
    assert np.abs(dt.cpu().numpy() - rdt).max() / np.abs(rdt).max() < _tol(l_max)
    assert np.abs(dh.cpu().numpy() - rdh).max() / np.abs(rdh).max() < _tol(l_max)


def test_ozaki_stage_is_deterministic_and_matches_fp64_plan():
    """Two calls give bit-identical outputs (the integer accumulation has no
    order dependence), and they agree with the FP64 plan's stage to 1e-10."""
    from magic_b200 import Plan

    l_max, N = 85, 5
    g = og.Grid(l_max)
    rng = np.random.default_rng(3)
    f = _fields(g, N, rng, True, False)
    prof = ostage.bouss_profiles(N, l_max=l_max)
    cu = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()
    fd = {k: cu(v) for k, v in f.items()}
    pd = {k: cu(v) for k, v in prof.items()}
    po, pf = Plan(l_max, precision="ozaki"), Plan(l_max)
    a, _, _ = po.nl_bouss(fd, pd, 200.0, 2.5, 1.0, 0.2)
    b, _, _ = po.nl_bouss(fd, pd, 200.0, 2.5, 1.0, 0.2)
    c, _, _ = pf.nl_bouss(fd, pd, 200.0, 2.5, 1.0, 0.2)
    torch.cuda.synchronize()
    po.poll_status(block=True)
    for k in a:
        assert torch.equal(a[k], b[k]), k
        scale = max(c[k].abs().max().item(), c[PAIR[k]].abs().max().item() if k in PAIR else 0)
        assert (a[k] - c[k]).abs().max().item() < _tol(l_max) * scale, k


def test_ozaki_plan_transforms_are_fp64():
    """Drop-in transforms on a digit-split plan run the FP64 kernels: a round
    trip recovers its input to FP64 rounding."""
    from magic_b200 import Plan

    p = Plan(48, precision="ozaki")
    g = torch.Generator().manual_seed(1)
    c = torch.randn(p.lm_max, 3, dtype=torch.complex128, generator=g).cuda()
    c[torch.as_tensor(p.lm2m == 0)] = c[torch.as_tensor(p.lm2m == 0)].real.to(c.dtype)
    back = p.scal_to_SH(p.scal_to_spat(c))
    torch.cuda.synchronize()
    assert (back - c).abs().max().item() < 1e-12 * c.abs().max().item()
