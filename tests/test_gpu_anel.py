"""GPU parity of the fused anelastic stages against the FP64 oracle
restatement of radial_loop_anel (magic_torch/step_time.py:1215-1475): the
split-precision stage (bf16x3 tcgen05 Legendre GEMMs, FP32 phi stage with
get_nl_anel, viscous and Ohmic heating), the digit-split stage (int8
digit-plane GEMMs, FP64 phi stage) and the FP64 composition.

Split tolerance: relative to the output's scale (the vector pair's max(|S|, |T|)
for the S/T outputs), 2e-5 up to l_max = 127 and 5e-5 above, as for the
Boussinesq stage; Courant steps 1e-5.  The l_max = 383 case (n_phi = 1152,
block FFT) is the anelastic benchmark configuration's resolution with a few
radial levels.  Measured on B200: 4e-7 to 1.5e-6 up to l_max = 42, up to
1.8e-5 (Advt) at l_max = 127 and 2.2e-5 at l_max = 383.
"""

import numpy as np
import pytest
import torch

from oracle import grid as og
from oracle import stage as ostage

pytestmark = pytest.mark.gpu

CASES = [
    (16, 1, 5, True, False),
    (32, 4, 6, True, True),
    (20, 1, 5, False, True),
    (42, 1, 4, False, False),
    (127, 1, 4, True, False),
    (255, 1, 3, True, True),
    (383, 1, 3, True, False),
]
PAIR = {"Advt": "Advp", "Advp": "Advt", "VxBt": "VxBp", "VxBp": "VxBt"}


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
def test_split_anel_stage_matches_oracle(l_max, minc, N, l_mag, l_chem):
    from magic_b200 import Plan

    g = og.Grid(l_max, minc)
    p = Plan(l_max, minc, precision="split")
    rng = np.random.default_rng(7 * l_max + N)
    f = _fields(g, N, rng, l_mag, l_chem)
    prof = ostage.anel_profiles(N, l_max=l_max)
    LF, vhf, ohm, cf, af, opm = 200.0, 0.3, 0.2, 2.5, 1.0, 0.2
    ref, rdt, rdh = ostage.nl_anel_stage(g, f, prof, LF, vhf, ohm, cf, af, opm, l_mag, l_chem)
    cu = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()
    work = torch.zeros(p.nl_anel_workspace(N, l_mag, l_chem), dtype=torch.uint8, device="cuda")
    out, dt, dh = p.nl_anel({k: cu(v) for k, v in f.items()}, {k: cu(v) for k, v in prof.items()},
                            LF, vhf, ohm, cf, af, opm, l_mag=l_mag, l_chem=l_chem, work=work)
    torch.cuda.synchronize()
    assert int(work[:4].view(torch.int32).item()) == 0, "device wait timed out"
    worst = {}
    for k in ref:
        got = out[k].cpu().numpy()
        assert np.all(got[:, 0] == 0) and np.all(got[:, -1] == 0), k
        scale = np.abs(ref[k]).max()
        if k in PAIR:
            scale = max(scale, np.abs(ref[PAIR[k]]).max())
        worst[k] = np.abs(got - ref[k]).max() / scale
    print("split anel stage errors", {k: f"{v:.2e}" for k, v in worst.items()})
    tol = 2e-5 if l_max <= 127 else 5e-5
    for k, v in worst.items():
        assert v < tol, (k, v)
    assert np.abs(dt.cpu().numpy() - rdt).max() / np.abs(rdt).max() < 1e-5
    assert np.abs(dh.cpu().numpy() - rdh).max() / np.abs(rdh).max() < 1e-5


FP64_CASES = [(16, 1, 5, True, False), (32, 4, 6, True, True), (383, 1, 3, True, False)]


@pytest.mark.parametrize("l_max,minc,N,l_mag,l_chem", FP64_CASES)
def test_fp64_anel_stage_matches_oracle(l_max, minc, N, l_mag, l_chem):
    """FP64 plans compose the anelastic stage from the FP64 kernels; the l_max = 383
    case is the anelastic configuration's horizontal grid (n_phi = 1152).  Tolerance
    1e-12 of each output's scale (the vector pair's for S/T) up to l_max 127, 4e-12
    on the 576 x 1152 grid, where each analysed coefficient sums ~7e5 products of
    mixed sign (measured 1.1e-12 in Advt; FP64 rounding of two summation orders)."""
    from magic_b200 import Plan

    g = og.Grid(l_max, minc)
    p = Plan(l_max, minc)
    rng = np.random.default_rng(11 * l_max + N)
    f = _fields(g, N, rng, l_mag, l_chem)
    prof = ostage.anel_profiles(N, l_max=l_max)
    LF, vhf, ohm, cf, af, opm = 200.0, 0.3, 0.2, 2.5, 1.0, 0.2
    ref, rdt, rdh = ostage.nl_anel_stage(g, f, prof, LF, vhf, ohm, cf, af, opm, l_mag, l_chem)
    cu = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()
    out, dt, dh = p.nl_anel({k: cu(v) for k, v in f.items()}, {k: cu(v) for k, v in prof.items()},
                            LF, vhf, ohm, cf, af, opm, l_mag=l_mag, l_chem=l_chem)
    torch.cuda.synchronize()
    assert set(out) == set(ref)
    tol = 1e-12 if l_max <= 127 else 4e-12
    for k in ref:
        got = out[k].cpu().numpy()
        assert np.all(got[:, 0] == 0) and np.all(got[:, -1] == 0), k
        scale = np.abs(ref[k]).max()
        if k in PAIR:
            scale = max(scale, np.abs(ref[PAIR[k]]).max())
        assert np.abs(got - ref[k]).max() / scale < tol, k
    assert np.abs(dt.cpu().numpy() - rdt).max() / np.abs(rdt).max() < 1e-12
    assert np.abs(dh.cpu().numpy() - rdh).max() / np.abs(rdh).max() < 1e-12


OZAKI_CASES = [
    (16, 1, 5, True, False),
    (32, 4, 6, True, True),
    (20, 1, 5, False, True),
    (42, 1, 4, False, False),
    (255, 1, 3, True, True),
    (383, 1, 3, False, False),
    (383, 1, 3, True, False),
]


@pytest.mark.parametrize("l_max,minc,N,l_mag,l_chem", OZAKI_CASES)
def test_ozaki_anel_stage_matches_oracle(l_max, minc, N, l_mag, l_chem):
    """Digit-split (ozaki) plans fuse the anelastic stage: the split stage's row
    programs on the int8 digit-plane GEMMs and the FP64 phi kernel k_nl_anel_f64.
    Tolerance 5e-13 l_max^2 of each output's scale, as for the digit-split
    Boussinesq stage (the digits keep 41 bits of each operand row's largest value;
    the analysis rows' 1/sin^2 weight makes the polar rows the largest); Courant
    steps likewise.  The l_max = 383 case is the anelastic configuration's grid
    (n_theta 576, n_phi 1152, block FFT).  Measured on B200: 2e-12 ... 4.4e-11
    up to l_max = 42, 2.1e-8 (Advt; bound 3.3e-8) at l_max = 255, 8.7e-10 (VSr)
    at l_max = 383; heat 1.3e-12 ... 2.8e-12 throughout."""
    from magic_b200 import Plan

    g = og.Grid(l_max, minc)
    p = Plan(l_max, minc, precision="ozaki")
    need = p.nl_anel_workspace(N, l_mag, l_chem)
    assert need > 0, "the fused digit-split stage should cover this grid"
    rng = np.random.default_rng(13 * l_max + N)
    f = _fields(g, N, rng, l_mag, l_chem)
    prof = ostage.anel_profiles(N, l_max=l_max)
    LF, vhf, ohm, cf, af, opm = 200.0, 0.3, 0.2, 2.5, 1.0, 0.2
    ref, rdt, rdh = ostage.nl_anel_stage(g, f, prof, LF, vhf, ohm, cf, af, opm, l_mag, l_chem)
    cu = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()
    work = torch.zeros(need, dtype=torch.uint8, device="cuda")
    out, dt, dh = p.nl_anel({k: cu(v) for k, v in f.items()}, {k: cu(v) for k, v in prof.items()},
                            LF, vhf, ohm, cf, af, opm, l_mag=l_mag, l_chem=l_chem, work=work)
    torch.cuda.synchronize()
    assert p.device_status(work) == 0, "device wait timed out"
    assert set(out) == set(ref)
    tol = 5e-13 * l_max ** 2
    worst = {}
    for k in ref:
        got = out[k].cpu().numpy()
        assert np.all(got[:, 0] == 0) and np.all(got[:, -1] == 0), k
        scale = np.abs(ref[k]).max()
        if k in PAIR:
            scale = max(scale, np.abs(ref[PAIR[k]]).max())
        worst[k] = np.abs(got - ref[k]).max() / scale
    print("ozaki anel stage errors", {k: f"{v:.2e}" for k, v in worst.items()})
    for k, v in worst.items():
        assert v < tol, (k, v)
    assert np.abs(dt.cpu().numpy() - rdt).max() / np.abs(rdt).max() < tol
    assert np.abs(dh.cpu().numpy() - rdh).max() / np.abs(rdh).max() < tol

