"""Split-precision drop-in transforms (bf16x3 tcgen05 Legendre GEMMs, FP32 phi
stage) against the FP64 oracle, and the synthesis -> analysis round trip of
the standalone SHT benchmark configuration (l_max = 127, 65 levels x (1
scalar + 2 torpol vector fields)).

Tolerances are relative to each output's (or vector pair's) largest value:
2e-5 for the transforms (FP32 Fourier rows, FP32 FFT, FP32 tensor-core
accumulation), and 1e-5 for the round trip of smooth |c_lm| ~ (l+1)^-2
spectra.  Measured on B200: 1.5e-7 to 1e-6 up to l_max = 127, up to 2.6e-6
(scal_to_SH) at l_max = 255; round trip 2.1e-6 (scalar, Q) and 6e-7 (S, T).
"""

import numpy as np
import pytest
import torch

from oracle import grid as og
from oracle import sht as osht

pytestmark = pytest.mark.gpu

cu = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()
npy = lambda t: t.cpu().numpy()


def _err(a, b, scale=None):
    return np.abs(a - b).max() / (np.abs(b).max() if scale is None else scale)


def _spec(rng, g, B, ex=1.5):
    x = (rng.standard_normal((g.lm_max, B)) + 1j * rng.standard_normal((g.lm_max, B)))
    x *= ((g.lm2l + 1.0) ** -ex)[:, None]
    x[g.lm2m == 0] = x[g.lm2m == 0].real
    return x


# n_phi 48 / 24 / 60 (block FFT), 384 / 768 (half-warp FFT)
@pytest.mark.parametrize("l_max,minc,B", [(16, 1, 3), (32, 4, 5), (20, 1, 4), (127, 1, 7),
                                          (255, 1, 3)])
def test_split_transforms_match_oracle(l_max, minc, B):
    from magic_b200 import Plan

    g = og.Grid(l_max, minc)
    p = Plan(l_max, minc, precision="split")
    rng = np.random.default_rng(3 * l_max + B)
    X = _spec(rng, g, B)
    Q, S, T = (_spec(rng, g, B) for _ in range(3))
    errs = {}
    errs["scal_to_spat"] = _err(npy(p.scal_to_spat(cu(X))), osht.scal_to_spat(g, X))
    ours = p.torpol_to_spat(cu(Q), cu(S), cu(T))
    ref = osht.torpol_to_spat(g, Q, S, T)
    errs["torpol r"] = _err(npy(ours[0]), ref[0])
    vs = max(np.abs(ref[1]).max(), np.abs(ref[2]).max())
    errs["torpol t"] = _err(npy(ours[1]), ref[1], vs)
    errs["torpol p"] = _err(npy(ours[2]), ref[2], vs)
    gt, gp = p.scal_to_grad_spat(cu(X))
    rt, rp = osht.scal_to_grad_spat(g, X)
    gs = max(np.abs(rt).max(), np.abs(rp).max())
    errs["grad"] = max(_err(npy(gt), rt, gs), _err(npy(gp), rp, gs))
    # analysis of band-limited grids (synthesised by the oracle)
    grid = osht.scal_to_spat(g, X)
    errs["scal_to_SH"] = _err(npy(p.scal_to_SH(cu(grid))), osht.scal_to_SH(g, grid))
    s, t = p.spat_to_sphertor(cu(ref[1]), cu(ref[2]))
    rs, rt2 = osht.spat_to_sphertor(g, ref[1], ref[2])
    st = max(np.abs(rs).max(), np.abs(rt2).max())
    errs["sphertor S"] = _err(npy(s), rs, st)
    errs["sphertor T"] = _err(npy(t), rt2, st)
    print("split transform errors", {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < 2e-5, (k, v)


def test_split_roundtrip_sht_benchmark_config():
    """l_max = 127, 65 levels x (1 scalar + 2 torpol): |c_lm| ~ (l+1)^-2 with
    seeded uniform phases, m = 0 real; synthesis then analysis recovers the
    input (Gauss-Legendre quadrature is exact for these degrees)."""
    from magic_b200 import Plan

    p = Plan(127, 1, precision="split")
    B = 65
    gen = torch.Generator(device="cpu").manual_seed(0)
    l = torch.as_tensor(p.lm2l, dtype=torch.float64)
    m0 = torch.as_tensor(p.lm2m == 0)

    def spec():
        ph = torch.rand(p.lm_max, B, generator=gen, dtype=torch.float64) * 2 * np.pi
        c = torch.polar((l + 1.0)[:, None] ** -2 * torch.ones(1, B, dtype=torch.float64), ph)
        c[m0] = c[m0].real.to(c.dtype)
        return c.cuda()

    c, Q, S, T = spec(), spec(), spec(), spec()
    back = p.scal_to_SH(p.scal_to_spat(c))
    e_s = ((back - c).abs().max() / c.abs().max()).item()
    br, bt, bp = p.torpol_to_spat(Q, S, T)
    q2 = p.scal_to_SH(br)
    s2, t2 = p.spat_to_sphertor(bt, bp)
    lpos = torch.as_tensor(p.lm2l > 0).cuda()
    e_q = ((q2 - Q).abs().max() / Q.abs().max()).item()
    e_st = max(((s2 - S)[lpos].abs().max() / S.abs().max()).item(),
               ((t2 - T)[lpos].abs().max() / T.abs().max()).item())
    print(f"split round trip: scalar {e_s:.1e}, Q {e_q:.1e}, S/T {e_st:.1e}")
    assert e_s < 1e-5 and e_q < 1e-5 and e_st < 1e-5


@pytest.mark.parametrize("name", ["sht_l16", "sht_l32m4", "sht_l64"])
def test_reference_signature_module_split(name):
    """The module-level drop-in (magic_b200.sht, reference signatures) on a
    split-precision plan against the reference's own golden outputs: 1-D and
    batched inputs, every helper, relative error below 2e-5."""
    import magic_b200
    from magic_b200 import sht
    from conftest import load_golden, rel_err

    z = load_golden(name)
    magic_b200.configure({"l_max": int(z["l_max"]), "minc": int(z["minc"]), "precision": "split"})
    try:
        tol = 2e-5
        assert rel_err(npy(sht.pol_to_curlr_spat(cu(z["Q"]))), z["curlr"]) < tol
        dt, dp = sht.torpol_to_dphspat(cu(z["S"][:, 0]), cu(z["T"][:, 0]))
        assert rel_err(npy(dt), z["dph_t"]) < tol and rel_err(npy(dp), z["dph_p"]) < tol
        cr, ct, cp = sht.torpol_to_curl_spat(cu(z["or2"]), cu(z["Bl"]), cu(z["ddB"]),
                                             cu(z["J"]), cu(z["dJ"]))
        assert rel_err(npy(cr), z["curl_r"]) < tol
        assert rel_err(npy(ct), z["curl_t"]) < tol and rel_err(npy(cp), z["curl_p"]) < tol
        vt, vp = sht.sphtor_to_spat(cu(z["S"][:, 0]), cu(z["T"][:, 0]))
        assert rel_err(npy(vt), z["sphtor_t"]) < tol and rel_err(npy(vp), z["sphtor_p"]) < tol
        q, s, t = sht.spat_to_qst(cu(z["grid"][0]), cu(z["vt"][0]), cu(z["vp"][0]))
        assert rel_err(npy(q), z["qst_q"]) < tol
        assert rel_err(npy(s), z["qst_s"]) < tol and rel_err(npy(t), z["qst_t"]) < tol
    finally:
        magic_b200.configure({})
