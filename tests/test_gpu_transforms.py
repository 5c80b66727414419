"""GPU parity of the FP64 transforms against the reference golden vectors and the oracle.

Tolerance (plain FP64 mode): 1e-12 normwise relative (max|a-b| / max|b|).
"""

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err
from oracle import grid as og
from oracle import sht as osht

pytestmark = pytest.mark.gpu

SHT = ["sht_l16", "sht_l32m4", "sht_l20", "sht_l31m2", "sht_l64"]
TOL = 1e-12
_plans = {}


def plan(l_max, minc=1):
    from magic_b200 import Plan

    key = (l_max, minc)
    if key not in _plans:
        _plans[key] = Plan(l_max, minc)
    return _plans[key]


def cu(x):
    return torch.as_tensor(np.ascontiguousarray(x)).cuda()


def npy(x):
    return x.detach().cpu().numpy()


@pytest.mark.parametrize("name", [n for n in SHT if n != "sht_l64"])
def test_tables_match_reference(name):
    z = load_golden(name)
    p = plan(int(z["l_max"]), int(z["minc"]))
    t = {k: npy(v) for k, v in p.tables().items()}
    assert rel_err(t["theta_ord"], z["theta_ord"]) < 1e-14
    assert rel_err(t["gauss"], z["gauss"]) < 1e-13
    assert rel_err(t["Plm"], z["Plm"]) < 1e-13
    assert rel_err(t["dPlm"], z["dPlm"]) < 1e-13


@pytest.mark.parametrize("name", SHT)
def test_transforms_match_reference(name):
    z = load_golden(name)
    p = plan(int(z["l_max"]), int(z["minc"]))
    assert rel_err(npy(p.scal_to_spat(cu(z["Slm"]))), z["scal_to_spat"]) < TOL
    assert rel_err(npy(p.scal_to_spat(cu(z["Slm"][:, 0]))), z["scal_to_spat_1d"]) < TOL
    assert rel_err(npy(p.scal_to_SH(cu(z["grid"]))), z["scal_to_SH"]) < TOL
    assert rel_err(npy(p.scal_to_SH(cu(z["grid"][0]))), z["scal_to_SH_1d"]) < TOL
    br, bt, bp = p.torpol_to_spat(cu(z["Q"]), cu(z["S"]), cu(z["T"]))
    assert rel_err(npy(br), z["torpol_br"]) < TOL
    assert rel_err(npy(bt), z["torpol_bt"]) < TOL
    assert rel_err(npy(bp), z["torpol_bp"]) < TOL
    s, t = p.spat_to_sphertor(cu(z["vt"]), cu(z["vp"]))
    assert rel_err(npy(s), z["sphertor_S"]) < TOL
    assert rel_err(npy(t), z["sphertor_T"]) < TOL
    gt, gp = p.scal_to_grad_spat(cu(z["Slm"]))
    assert rel_err(npy(gt), z["grad_t"]) < TOL and rel_err(npy(gp), z["grad_p"]) < TOL
    pt, pp = p.pol_to_grad_spat(cu(z["S"]))
    assert rel_err(npy(pt), z["polgrad_t"]) < TOL and rel_err(npy(pp), z["polgrad_p"]) < TOL
    e10 = np.zeros(int(z["lm_max"]), dtype=np.complex128)
    e10[1] = 1.0
    y10 = npy(p.scal_to_spat(cu(e10)))
    assert rel_err(y10, z["y10"]) < TOL
    assert y10[0::2].mean() > 0 > y10[1::2].mean()  # Y_1^0 > 0 in the north


@pytest.mark.parametrize("name", ["sht_l16", "sht_l32m4", "sht_l64"])
def test_reference_signature_module(name):
    import magic_b200
    from magic_b200 import sht

    z = load_golden(name)
    magic_b200.configure({"l_max": int(z["l_max"]), "minc": int(z["minc"])})
    assert rel_err(npy(sht.pol_to_curlr_spat(cu(z["Q"]))), z["curlr"]) < TOL
    dt, dp = sht.torpol_to_dphspat(cu(z["S"][:, 0]), cu(z["T"][:, 0]))
    assert rel_err(npy(dt), z["dph_t"]) < TOL and rel_err(npy(dp), z["dph_p"]) < TOL
    cr, ct, cp = sht.torpol_to_curl_spat(cu(z["or2"]), cu(z["Bl"]), cu(z["ddB"]), cu(z["J"]),
                                         cu(z["dJ"]))
    assert rel_err(npy(cr), z["curl_r"]) < TOL
    assert rel_err(npy(ct), z["curl_t"]) < TOL and rel_err(npy(cp), z["curl_p"]) < TOL
    vt, vp = sht.sphtor_to_spat(cu(z["S"][:, 0]), cu(z["T"][:, 0]))
    assert rel_err(npy(vt), z["sphtor_t"]) < TOL and rel_err(npy(vp), z["sphtor_p"]) < TOL
    q, s, t = sht.spat_to_qst(cu(z["grid"][0]), cu(z["vt"][0]), cu(z["vp"][0]))
    assert rel_err(npy(q), z["qst_q"]) < TOL
    assert rel_err(npy(s), z["qst_s"]) < TOL and rel_err(npy(t), z["qst_t"]) < TOL


def _spec(rng, g, B, decay=2.0, real_m0=True):
    amp = (g.lm2l + 1.0) ** (-decay)
    x = (rng.standard_normal((g.lm_max, B)) + 1j * rng.standard_normal((g.lm_max, B)))
    x *= amp[:, None]
    if real_m0:
        x[g.lm2m == 0] = x[g.lm2m == 0].real
    return x


@pytest.mark.parametrize("l_max,minc,B", [(127, 1, 7), (85, 1, 3), (48, 3, 9)])
def test_against_oracle(l_max, minc, B):
    """Random coefficients at sizes the oracle finishes in seconds."""
    g = og.Grid(l_max, minc)
    p = plan(l_max, minc)
    rng = np.random.default_rng(l_max)
    X = _spec(rng, g, B, real_m0=False)
    Q, S, T = (_spec(rng, g, B) for _ in range(3))
    assert rel_err(npy(p.scal_to_spat(cu(X))), osht.scal_to_spat(g, X)) < TOL
    ours = p.torpol_to_spat(cu(Q), cu(S), cu(T))
    ref = osht.torpol_to_spat(g, Q, S, T)
    for a, b in zip(ours, ref):
        assert rel_err(npy(a), b) < TOL
    grid = rng.standard_normal((B, g.n_theta_max, g.n_phi_max))
    assert rel_err(npy(p.scal_to_SH(cu(grid))), osht.scal_to_SH(g, grid)) < TOL
    vt = rng.standard_normal((B, g.n_theta_max, g.n_phi_max))
    s, t = p.spat_to_sphertor(cu(grid), cu(vt))
    rs, rt = osht.spat_to_sphertor(g, grid, vt)
    assert rel_err(npy(s), rs) < TOL and rel_err(npy(t), rt) < TOL


@pytest.mark.parametrize("l_max,B", [(255, 97), (383, 12)])
def test_roundtrip_full_size(l_max, B):
    """Size-independent properties at the benchmark resolutions: Gauss-Legendre
    quadrature integrates P_lm P_l'm exactly, so analysis(synthesis(c)) == c."""
    from magic_b200 import Plan

    p = Plan(l_max)
    g = torch.Generator(device="cpu").manual_seed(0)
    l = torch.as_tensor(p.lm2l, dtype=torch.float64)
    m0 = torch.as_tensor(p.lm2m == 0)
    phase = torch.rand(p.lm_max, B, generator=g, dtype=torch.float64) * 2 * np.pi
    c = torch.polar((l + 1.0)[:, None] ** -2 * torch.ones(1, B, dtype=torch.float64), phase)
    c[m0] = c[m0].real.to(c.dtype)
    c = c.cuda()
    back = p.scal_to_SH(p.scal_to_spat(c))
    assert (back - c).abs().max().item() / c.abs().max().item() < 1e-12
    # vector: torpol -> (bt, bp) -> sphertor recovers S, T for l >= 1; br -> Q
    S = c.clone()
    T = torch.roll(c, 1, dims=1)
    Q = torch.roll(c, 2, dims=1)
    br, bt, bp = p.torpol_to_spat(Q, S, T)
    s2, t2 = p.spat_to_sphertor(bt, bp)
    q2 = p.scal_to_SH(br)
    lpos = torch.as_tensor(p.lm2l > 0).cuda()
    assert (s2 - S)[lpos].abs().max().item() / S.abs().max().item() < 1e-12
    assert (t2 - T)[lpos].abs().max().item() / T.abs().max().item() < 1e-12
    assert (q2 - Q).abs().max().item() / Q.abs().max().item() < 1e-12
    # linearity of synthesis
    a, b = 0.37, -1.9
    lhs = p.scal_to_spat(a * c + b * S.flip(1))
    rhs = a * p.scal_to_spat(c) + b * p.scal_to_spat(S.flip(1))
    assert (lhs - rhs).abs().max().item() / rhs.abs().max().item() < 1e-13


def test_errors_are_loud():
    from magic_b200 import Plan
    from magic_b200._lib import MagicError

    p = plan(16)
    with pytest.raises(ValueError):
        p.scal_to_spat(torch.zeros(10, dtype=torch.complex128, device="cuda"))
    with pytest.raises(ValueError):
        p.scal_to_SH(torch.zeros(2, 3, 4, dtype=torch.float64, device="cuda"))
    with pytest.raises(MagicError):
        Plan(16, n_theta_max=25)  # odd theta count
    with pytest.raises(MagicError):
        Plan(900)  # n_phi above the shared-memory FFT limit
