"""Spectral explicit terms (get_td + finish_exp) and radial operators on the
GPU, in FP64: against the reference's own outputs (tests/golden/td_*.npz),
against the numpy oracle at larger sizes, and through size-independent
properties at the l_max = 255, n_r = 97 finite-difference configuration.

Tolerance: 1e-12 relative to each output's largest value (FP64; the kernels
fuse multiply-adds where the reference rounds products separately, and the
dense Chebyshev operator sums in a different order than the reference's
matrix product).
"""

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err
from oracle import td as otd

pytestmark = pytest.mark.gpu

TOL = 1e-12
cu = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()
npy = lambda t: t.cpu().numpy()
PROF = ("r", "or1", "or2", "or4", "orho1", "beta")


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
@pytest.mark.parametrize("dc", [False, True])
def test_get_td_matches_reference(name, dc):
    from magic_b200 import Plan
    from magic_b200.radial import RadialOp

    z = load_golden(name)
    p = Plan(int(z["l_max"]), int(z["minc"]))
    assert p.lm_max == int(z["lm_max"])
    D1 = RadialOp(z["D1"])
    ins = {k[3:]: cu(z[k]) for k in z if k.startswith("in_")}
    prof = {k: cu(z[k]) for k in PROF}
    o = p.get_td(ins, prof, float(z["CorFac"]), D1, l_double_curl=dc, l_heat=True, l_mag=True,
                 l_chem=True, l_anel=bool(z["l_anel"]))
    errs = {"dwdt": rel_err(npy(o["dwdt"]), z["dwdt_dc_fin"] if dc else z["dwdt"])}
    if not dc:
        errs["dpdt"] = rel_err(npy(o["dpdt"]), z["dpdt"])
    for k in ("dzdt", "dsdt", "dxidt", "dbdt", "djdt"):
        errs[k] = rel_err(npy(o[k]), z[k])
    print(name, "double curl" if dc else "standard", {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < TOL, (k, v)


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
def test_radial_ops_match_reference(name):
    from magic_b200.radial import RadialOp, costf, get_ddr, get_dr

    z = load_golden(name)
    D1, D2 = RadialOp(z["D1"]), RadialOp(z["D2"])
    n_r = int(z["n_r_max"])
    assert D1.bandwidth == (n_r if name == "td_cheb" else 5)
    f = cu(z["in_f"])
    assert rel_err(npy(get_dr(f, D1)), z["dr_f"]) < TOL
    d1, d2 = get_ddr(f, D1, D2)
    assert rel_err(npy(d1), z["ddr_f1"]) < TOL and rel_err(npy(d2), z["ddr_f2"]) < TOL
    c = costf(f)
    assert rel_err(npy(c), z["costf_f"]) < TOL
    assert rel_err(npy(costf(c)), z["in_f"]) < TOL  # self-inverse


def _random_case(p, n_r, r, seed, anel):
    rng = np.random.default_rng(seed)
    lm = p.lm_max
    amp = (p.lm2l.astype(np.float64) + 1.0)[:, None] ** -1.0

    def spec():
        return (rng.standard_normal((lm, n_r)) + 1j * rng.standard_normal((lm, n_r))) * amp

    names = ["Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt", "VxBp", "VXir", "VXit",
             "w", "dw", "ddw", "z", "dz"]
    ins = {k: spec() for k in names}
    prof = dict(r=r, or1=1.0 / r, or2=1.0 / r ** 2, or4=1.0 / r ** 4,
                orho1=np.exp(-0.5 * (r - r[-1])) if anel else np.ones(n_r),
                beta=-0.5 * np.ones(n_r) if anel else np.zeros(n_r))
    return ins, prof


@pytest.mark.parametrize("scheme,l_max,n_r", [("chebyshev", 127, 65), ("FD", 255, 97)])
def test_get_td_vs_oracle(scheme, l_max, n_r):
    """Every output against the numpy oracle on seeded inputs at the standalone-SHT
    size (Chebyshev, l_max = 127, 65 levels) and at the l_max = 255, n_r = 97
    fourth-order finite-difference configuration, both poloidal forms."""
    from magic_b200 import Plan
    from magic_b200.radial import RadialScheme

    p = Plan(l_max, 1)
    sch = RadialScheme(n_r, scheme, fd_order=4 if scheme == "FD" else 2)
    anel = scheme == "FD"
    ins, prof = _random_case(p, n_r, sch.r, l_max, anel)
    g = dict(lm2l=p.lm2l, lm2m=p.lm2m, l_max=l_max, CorFac=1e5, l_anel=int(anel), **prof)
    dins = {k: cu(v) for k, v in ins.items()}
    dprof = {k: cu(v) for k, v in prof.items()}
    for dc in (0, 1):
        g["l_double_curl"] = dc
        ref = otd.get_td(g, ins, sch.D1m)
        o = p.get_td(dins, dprof, 1e5, sch.D1, l_double_curl=bool(dc), l_heat=True, l_mag=True,
                     l_chem=True, l_anel=anel)
        for k in o:
            e = rel_err(npy(o[k]), ref[k])
            assert e < TOL, (scheme, dc, k, e)


@pytest.mark.parametrize("scheme", ["chebyshev", "FD"])
def test_radial_derivative_of_quadratic_is_exact(scheme):
    """Size-independent property at l_max = 255, n_r = 97: both schemes differentiate
    a + b r + c r^2 exactly (Chebyshev for any polynomial of degree < n_r, the
    fourth-order finite differences and their second-order boundary rows for
    degree <= 2), per lm row, to rounding: |D f - f'| <= 16 eps ||D||_inf max|f|
    (the Chebyshev second-derivative operator has ||D2|| ~ 1e8 at 97 points)."""
    from magic_b200 import Plan
    from magic_b200.radial import RadialScheme, get_ddr

    p = Plan(255, 1)
    n_r = 97
    sch = RadialScheme(n_r, scheme, fd_order=4 if scheme == "FD" else 2)
    g = torch.Generator(device="cpu").manual_seed(5)
    abc = torch.randn(3, p.lm_max, 1, dtype=torch.complex128, generator=g).cuda()
    r = torch.as_tensor(sch.r).cuda()[None, :]
    f = abc[0] + abc[1] * r + abc[2] * r * r
    d1, d2 = get_ddr(f, sch.D1, sch.D2)
    eps = np.finfo(np.float64).eps
    fmax = f.abs().amax(dim=1)
    for d, exact, M in ((d1, abc[1] + 2 * abc[2] * r, sch.D1m), (d2, 2 * abc[2] + 0 * r, sch.D2m)):
        bound = 16 * eps * np.abs(M).sum(axis=1).max() * fmax
        err = (d - exact).abs().amax(dim=1)
        assert bool((err <= bound).all()), (scheme, (err / bound).max().item())
