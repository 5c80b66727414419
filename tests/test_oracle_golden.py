"""Pin the CPU oracle against golden vectors produced by the reference itself.

Tolerance: 1e-12 normwise relative (both sides FP64; differences are rounding
order only).  Tables are pinned at 1e-13.
"""

import numpy as np
import pytest

from conftest import load_golden, rel_err
from oracle import grid as og
from oracle import nonlinear as onl
from oracle import sht as osht

SHT = ["sht_l16", "sht_l32m4", "sht_l20", "sht_l31m2", "sht_l64"]
TOL = 1e-12

_grids = {}


def _grid(z):
    key = (int(z["l_max"]), int(z["minc"]))
    if key not in _grids:
        _grids[key] = og.Grid(*key)
    return _grids[key]


@pytest.mark.parametrize("name", SHT)
def test_sizes(name):
    z = load_golden(name)
    s = og.grid_sizes(int(z["l_max"]), int(z["minc"]))
    for k in ("lm_max", "n_theta_max", "n_phi_max", "n_m_max"):
        assert s[k] == int(z[k]), k


@pytest.mark.parametrize("name", [n for n in SHT if n != "sht_l64"])
def test_tables(name):
    z = load_golden(name)
    g = _grid(z)
    assert rel_err(g.theta_ord, z["theta_ord"]) < 1e-14
    assert rel_err(g.gauss, z["gauss"]) < 1e-13
    for k in ("Plm", "dPlm", "wPlm", "wdPlm"):
        assert rel_err(getattr(g, k), z[k]) < 1e-13, k
    assert rel_err(g.O_sin_theta_E2_grid, z["O_sin_theta_E2_grid"]) < 1e-13
    assert rel_err(g.cosn_theta_E2_grid, z["cosn_theta_E2_grid"]) < 1e-13


@pytest.mark.parametrize("name", SHT)
def test_scalar(name):
    z = load_golden(name)
    g = _grid(z)
    assert rel_err(osht.scal_to_spat(g, z["Slm"]), z["scal_to_spat"]) < TOL
    assert rel_err(osht.scal_to_spat(g, z["Slm"][:, 0]), z["scal_to_spat_1d"]) < TOL
    assert rel_err(osht.scal_to_SH(g, z["grid"]), z["scal_to_SH"]) < TOL
    assert rel_err(osht.scal_to_SH(g, z["grid"][0]), z["scal_to_SH_1d"]) < TOL
    assert rel_err(osht.scal_to_spat(g, np.eye(1, int(z["lm_max"]), 1)[0].astype(complex)),
                   z["y10"]) < TOL


@pytest.mark.parametrize("name", SHT)
def test_vector(name):
    z = load_golden(name)
    g = _grid(z)
    br, bt, bp = osht.torpol_to_spat(g, z["Q"], z["S"], z["T"])
    assert rel_err(br, z["torpol_br"]) < TOL
    assert rel_err(bt, z["torpol_bt"]) < TOL
    assert rel_err(bp, z["torpol_bp"]) < TOL
    br, bt, bp = osht.torpol_to_spat(g, z["Q"][:, 0], z["S"][:, 0], z["T"][:, 0])
    assert rel_err(bt, z["torpol1_bt"]) < TOL and rel_err(bp, z["torpol1_bp"]) < TOL
    s, t = osht.spat_to_sphertor(g, z["vt"], z["vp"])
    assert rel_err(s, z["sphertor_S"]) < TOL
    assert rel_err(t, z["sphertor_T"]) < TOL
    s, t = osht.spat_to_sphertor(g, z["vt"][0], z["vp"][0])
    assert rel_err(s, z["sphertor1_S"]) < TOL and rel_err(t, z["sphertor1_T"]) < TOL


@pytest.mark.parametrize("name", SHT)
def test_helpers(name):
    z = load_golden(name)
    g = _grid(z)
    gt, gp = osht.scal_to_grad_spat(g, z["Slm"])
    assert rel_err(gt, z["grad_t"]) < TOL and rel_err(gp, z["grad_p"]) < TOL
    assert rel_err(osht.pol_to_curlr_spat(g, z["Q"]), z["curlr"]) < TOL
    pt, pp = osht.pol_to_grad_spat(g, z["S"])
    assert rel_err(pt, z["polgrad_t"]) < TOL and rel_err(pp, z["polgrad_p"]) < TOL
    dt, dp = osht.torpol_to_dphspat(g, z["S"][:, 0], z["T"][:, 0])
    assert rel_err(dt, z["dph_t"]) < TOL and rel_err(dp, z["dph_p"]) < TOL
    cr, ct, cp = osht.torpol_to_curl_spat(g, z["or2"], z["Bl"], z["ddB"], z["J"], z["dJ"])
    assert rel_err(cr, z["curl_r"]) < TOL
    assert rel_err(ct, z["curl_t"]) < TOL
    assert rel_err(cp, z["curl_p"]) < TOL
    vt, vp = osht.sphtor_to_spat(g, z["S"][:, 0], z["T"][:, 0])
    assert rel_err(vt, z["sphtor_t"]) < TOL and rel_err(vp, z["sphtor_p"]) < TOL
    q, s, t = osht.spat_to_qst(g, z["grid"][0], z["vt"][0], z["vp"][0])
    assert rel_err(q, z["qst_q"]) < TOL
    assert rel_err(s, z["qst_s"]) < TOL and rel_err(t, z["qst_t"]) < TOL


def test_get_nl():
    z = load_golden("nl_bouss")
    names = ["vr", "vt", "vp", "cvr", "cvt", "cvp", "s", "br", "bt", "bp",
             "cbr", "cbt", "cbp", "xi"]
    res = onl.get_nl(*[z[k] for k in names], z["or2"], z["or4"], z["ost2"], float(z["LFfac"]))
    onames = ["Advr", "Advt", "Advp", "VSr", "VSt", "VSp", "VxBr", "VxBt", "VxBp",
              "VXir", "VXit", "VXip"]
    for k, v in zip(onames, res):
        assert rel_err(v, z["out_" + k]) < 1e-14, k


def test_get_nl_anel():
    z = load_golden("nl_anel")
    names = ["vr", "vt", "vp", "dvrdr", "dvtdr", "dvpdr", "dvrdt", "dvrdp",
             "dvtdp", "dvpdp", "cvr", "s", "xi", "br", "bt", "bp", "cbr", "cbt", "cbp"]
    prof = [z[k] for k in ("r", "or1", "or2", "or4", "beta", "orho1", "otemp1",
                           "visc", "lambda_", "ost2", "cosn")]
    res = onl.get_nl_anel(*[z[k] for k in names], *prof, float(z["LFfac"]),
                          float(z["ViscHeatFac"]), float(z["OhmLossFac"]))
    onames = ["Advr", "Advt", "Advp", "VSr", "VSt", "VSp", "VxBr", "VxBt", "VxBp",
              "VXir", "VXit", "VXip", "heat"]
    assert float(z["OhmLossFac"]) != 0.0 and float(z["ViscHeatFac"]) != 0.0
    for k, v in zip(onames, res):
        assert rel_err(v, z["out_" + k]) < 1e-13, k


def test_courant():
    z = load_golden("nl_bouss")
    common = dict(courfac=float(z["courfac"]), alffac=float(z["alffac"]), or2=z["or2"],
                  or4=z["or4"], orho1=z["orho1"], orho2=z["orho2"], ost2=z["ost2"],
                  delxr2=z["delxr2"], delxh2=z["delxh2"], LFfac=float(z["LFfac"]),
                  opm=float(z["opm"]))
    r, h = onl.courant_check(z["vr"], z["vt"], z["vp"], z["br"], z["bt"], z["bp"], **common)
    assert rel_err(r, z["cour_damp_r"]) < 1e-14 and rel_err(h, z["cour_damp_h"]) < 1e-14
    r, h = onl.courant_check(z["vr"], z["vt"], z["vp"], None, None, None, **common)
    assert rel_err(r, z["cour_nomag_r"]) < 1e-14 and rel_err(h, z["cour_nomag_h"]) < 1e-14
    r, h = onl.courant_check(z["vr"], z["vt"], z["vp"], z["br"], z["bt"], z["bp"],
                             damp=False, **common)
    np.testing.assert_allclose(r, np.sqrt(z["delxr2"] / z["cour_nodamp_vr2"]), rtol=1e-14)
    np.testing.assert_allclose(h, np.sqrt(z["delxh2"] / z["cour_nodamp_vh2"]), rtol=1e-14)
    for case, ch, new in zip(z["dtc_cases"], z["dtc_changed"], z["dtc_new"]):
        c2, n2 = onl.dt_courant(*case)
        assert c2 == bool(ch) and n2 == new


def _td_setup(name):
    z = load_golden(name)
    g = {k: z[k] for k in ("lm2l", "lm2m", "r", "or1", "or2", "or4", "orho1", "beta")}
    g.update(l_max=int(z["l_max"]), CorFac=float(z["CorFac"]), l_anel=int(z["l_anel"]))
    ins = {k[3:]: z[k] for k in z if k.startswith("in_")}
    return z, g, ins


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
def test_td_oracle(name):
    """get_td + finish_exp restated in numpy against the reference's own outputs, in both
    poloidal forms (standard with dpdt, double curl with beta and 1/rho), plus the
    radial derivatives and the DCT-I."""
    from oracle import td

    z, g, ins = _td_setup(name)
    for dc in (0, 1):
        g["l_double_curl"] = dc
        o = td.get_td(g, ins, z["D1"])
        if dc:
            assert rel_err(o["dwdt"], z["dwdt_dc_fin"]) < 1e-14
        else:
            assert rel_err(o["dwdt"], z["dwdt"]) < 1e-14
            assert rel_err(o["dpdt"], z["dpdt"]) < 1e-14
        for k in ("dzdt", "dsdt", "dxidt", "dbdt", "djdt"):
            assert rel_err(o[k], z[k]) < 1e-14, k
    assert rel_err(td.radial_apply(z["D1"], z["in_f"]), z["dr_f"]) < 1e-14
    assert rel_err(td.radial_apply(z["D1"], z["in_f"]), z["ddr_f1"]) < 1e-14
    assert rel_err(td.radial_apply(z["D2"], z["in_f"]), z["ddr_f2"]) < 1e-14
    C = td.dct1_matrix(int(z["n_r_max"]))
    assert rel_err(td.radial_apply(C, z["in_f"]), z["costf_f"]) < 1e-14
    assert np.abs(C @ C - np.eye(C.shape[0])).max() < 1e-13  # self-inverse


def test_radial_scheme_builders():
    """The library's host-side Chebyshev and finite-difference builders reproduce the
    reference's grids and derivative matrices."""
    from magic_b200 import radial as R

    z = load_golden("td_cheb")
    r, D1, D2, _ = R.cheb_matrices(int(z["n_r_max"]))
    assert rel_err(r, z["r"]) < 1e-15
    assert rel_err(D1, z["D1"]) < 1e-13 and rel_err(D2, z["D2"]) < 1e-13
    z = load_golden("td_fd_anel")
    r = R.fd_grid(int(z["n_r_max"]))
    assert rel_err(r, z["r"]) < 1e-15
    D = R.fd_matrices(r, 4, 2)
    assert rel_err(D[0], z["D1"]) < 1e-13 and rel_err(D[1], z["D2"]) < 1e-13


def _s_case(name):
    z = load_golden(name)
    g = dict(lm2l=z["lm2l"], lm2m=z["lm2m"], l_max=int(z["l_max"]))
    prof = {k: z[k] for k in ("or1", "or2", "beta", "dLtemp0", "dLkappa", "kappa")}
    mats = (z["rMat"], z["drMat"], z["d2rMat"], float(z["rnorm"]), float(z["boundary_fac"]))
    st = dict(old=z["s_old"].copy(), impl=z["s_impl"].copy(), expl0=z["s_expl0"].copy(),
              expl1=z["s_expl1"].copy())
    return z, g, prof, mats, st


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
def test_update_s_oracle(name):
    """The implicit entropy update restated in numpy (per-l LU solves) against the
    reference's updateS (Chebyshev with the DCT-I; FD4 anelastic, where the reference
    uses a pivoted banded LU)."""
    from oracle import implicit as oi

    z, g, prof, mats, st = _s_case(name)
    w = (z["wimp"], z["wimp_lin"], z["wexp"])
    o = oi.update_s(g, mats, prof, st, w, float(z["opr"]), z["hdif_S"], z["tops"], z["bots"],
                    z["D1"], z["D2"], bool(z["chebyshev"]), int(z["n_cheb_max"]),
                    int(z["fd_order"]))
    assert rel_err(o["s"], z["s_new"]) < 1e-14
    assert rel_err(o["ds"], z["ds_new"]) < 1e-14
    assert rel_err(o["impl"], z["s_impl_new"]) < 1e-14
    assert rel_err(o["old"], z["s_old_new"]) < 1e-14
    assert rel_err(o["expl1"], z["s_expl1_new"]) == 0.0
    ref_w = oi.cnab2_weights(1e-4, 1.3e-4)
    assert np.allclose(ref_w[1], z["wimp_lin"], rtol=1e-15) and np.allclose(ref_w[2], z["wexp"],
                                                                            rtol=1e-15)


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
def test_scalar_solve_operators(name):
    """The library's host builder of the per-degree solve operators (inverse of the
    preconditioned LHS, DCT-I folded in for Chebyshev), applied in numpy, reproduces
    the reference's new field."""
    from types import SimpleNamespace

    from magic_b200 import implicit as I

    z = load_golden(name)
    sch = SimpleNamespace(n_r=int(z["n_r_max"]), chebyshev=bool(z["chebyshev"]),
                          n_cheb=int(z["n_cheb_max"]), rMat=z["rMat"], drMat=z["drMat"],
                          d2rMat=z["d2rMat"], rnorm=float(z["rnorm"]),
                          boundary_fac=float(z["boundary_fac"]))
    d1c = z["beta"] + z["dLtemp0"] + 2 * z["or1"] + z["dLkappa"]
    w = I.cnab2_weights(1e-4, 1.3e-4)
    M = I.scalar_solve_operators(sch, int(z["l_max"]), w[1], float(z["opr"]), z["hdif_S"],
                                 z["kappa"], d1c, z["or2"])
    rhs = w[0] * z["s_old"] + w[2] * z["s_impl"] + w[3] * z["s_expl0"] + w[4] * z["s_expl1"]
    rhs[:, 0] = z["tops"]
    rhs[:, -1] = z["bots"]
    x = np.stack([M[l] @ rhs[i] for i, l in enumerate(z["lm2l"])])
    x[z["lm2m"] == 0] = x[z["lm2m"] == 0].real
    assert rel_err(x, z["s_new"]) < 1e-13


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
def test_update_z_oracle(name):
    """The toroidal-velocity update restated in numpy against the reference's updateZ
    (Chebyshev with stress-free rows; FD4 anelastic with no-slip rows and the banded
    solve's identity at l = 0)."""
    from oracle import implicit as oi

    z = load_golden(name)
    g = dict(lm2l=z["lm2l"], lm2m=z["lm2m"], l_max=int(z["l_max"]))
    prof = {k: z[k] for k in ("or1", "or2", "beta", "dbeta", "dLvisc", "visc")}
    mats = (z["rMat"], z["drMat"], z["d2rMat"], float(z["rnorm"]), float(z["boundary_fac"]))
    st = {k: z["z_" + k].copy() for k in ("old", "impl", "expl0", "expl1")}
    o = oi.update_z(g, mats, prof, st, (z["wimp"], z["wimp_lin"], z["wexp"]), z["hdif_V"],
                    z["D1"], z["D2"], bool(z["chebyshev"]), int(z["n_cheb_max"]),
                    int(z["ktopv"]), int(z["kbotv"]), int(z["fd_order"]))
    for k, ref in (("x", "z_new"), ("dx", "dz_new"), ("impl", "z_impl_new"),
                   ("old", "z_old_new"), ("expl1", "z_expl1_new")):
        assert rel_err(o[k], z[ref]) < 1e-14, k


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
def test_toroidal_solve_operators(name):
    from types import SimpleNamespace

    from magic_b200 import implicit as I

    z = load_golden(name)
    sch = SimpleNamespace(n_r=int(z["n_r_max"]), chebyshev=bool(z["chebyshev"]),
                          n_cheb=int(z["n_cheb_max"]), rMat=z["rMat"], drMat=z["drMat"],
                          d2rMat=z["d2rMat"], rnorm=float(z["rnorm"]),
                          boundary_fac=float(z["boundary_fac"]), fd_order=int(z["fd_order"]))
    w = I.cnab2_weights(1e-4, 1.3e-4)
    M = I.toroidal_solve_operators(sch, int(z["l_max"]), w[1], z["hdif_V"], z["visc"], z["beta"],
                                   z["dbeta"], z["dLvisc"], z["or1"], z["or2"], int(z["ktopv"]),
                                   int(z["kbotv"]))
    rhs = w[0] * z["z_old"] + w[2] * z["z_impl"] + w[3] * z["z_expl0"] + w[4] * z["z_expl1"]
    rhs[:, 0] = 0.0
    rhs[:, -1] = 0.0
    if isinstance(M, I.Band):  # finite differences of order > 2: the banded LU solve
        from oracle import implicit as oi

        x = np.zeros_like(rhs)
        for l in range(int(z["l_max"]) + 1):
            rows = np.nonzero(z["lm2l"] == l)[0]
            abd, piv = oi.band_factor(M.A[l], M.kl, M.ku)
            y = oi.band_solve(abd, piv, M.kl, M.ku, (M.fr[l][None, :] * rhs[rows]).T).T
            x[rows] = y if M.fc is None else M.fc[l][None, :] * y
    else:
        x = np.stack([M[l] @ rhs[i] for i, l in enumerate(z["lm2l"])])
    x[z["lm2m"] == 0] = x[z["lm2m"] == 0].real
    assert rel_err(x, z["z_new"]) < 1e-13


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
def test_update_b_oracle(name):
    """The magnetic update (insulating inner core) restated in numpy against the
    reference's updateB, both fields and their first and second derivatives."""
    from oracle import implicit as oi

    z = load_golden(name)
    g = dict(lm2l=z["lm2l"], lm2m=z["lm2m"], l_max=int(z["l_max"]))
    prof = {k: z[k] for k in ("or1", "or2", "lambda_", "dLlambda")}
    mats = (z["rMat"], z["drMat"], z["d2rMat"], float(z["rnorm"]), float(z["boundary_fac"]))
    st = {f: {k: z[f + "_" + k].copy() for k in ("old", "impl", "expl0", "expl1")}
          for f in ("b", "j")}
    ob, oj = oi.update_b(g, mats, prof, st["b"], st["j"], (z["wimp"], z["wimp_lin"], z["wexp"]),
                         float(z["opm"]), z["hdif_B"], z["D1"], z["D2"], bool(z["chebyshev"]),
                         int(z["n_cheb_max"]), int(z["fd_order"]))
    for f, o in (("b", ob), ("j", oj)):
        for k, ref in (("x", f + "_new"), ("dx", "d" + f + "_new"), ("d2x", "dd" + f + "_new"),
                       ("impl", f + "_impl_new"), ("old", f + "_old_new"),
                       ("expl1", f + "_expl1_new")):
            assert rel_err(o[k], z[ref]) < 1e-14, (f, k)


def test_update_w_oracle():
    """The double-curl poloidal update with the l = 0 pressure restated in numpy
    against the reference's updateW (FD4 anelastic, no-slip)."""
    from oracle import implicit as oi

    z = load_golden("td_fd_anel")
    g = dict(lm2l=z["lm2l"], lm2m=z["lm2m"], l_max=int(z["l_max"]))
    prof = {k: z[k] for k in ("or1", "or2", "beta", "dbeta", "ddbeta", "visc", "dLvisc",
                              "ddLvisc", "orho1", "rgrav", "rho0")}
    mats = (z["rMat"], z["drMat"], z["d2rMat"], z["d3rMat"], z["d4rMat"])
    st = {k: z["w_" + k].copy() for k in ("old", "impl", "expl0", "expl1")}
    o = oi.update_w(g, mats, prof, st, (z["wimp"], z["wimp_lin"], z["wexp"]), z["hdif_V"],
                    z["D1"], z["D2"], z["s_new"], float(z["BuoFac"]), z["r"], int(z["fd_order"]),
                    int(z["ktopv"]), int(z["kbotv"]))
    for k, ref in (("x", "w_new"), ("dx", "dw_new"), ("d2x", "ddw_new"), ("impl", "w_impl_new"),
                   ("old", "w_old_new"), ("expl1", "w_expl1_new"), ("p0", "p0_new")):
        assert rel_err(o[k], z[ref]) < 1e-13, k


def _wp_case():
    z = load_golden("td_cheb")
    g = dict(lm2l=z["lm2l"], lm2m=z["lm2m"], l_max=int(z["l_max"]))
    prof = {k: z[k] for k in ("or1", "or2", "beta", "dbeta", "visc", "dLvisc", "rgrav", "rho0")}
    mats = (z["rMat"], z["drMat"], z["d2rMat"], float(z["rnorm"]), float(z["boundary_fac"]))
    stw = {k: z["wp_w_" + k].copy() for k in ("old", "impl", "expl0", "expl1")}
    stp = {k: z["wp_p_" + k].copy() for k in ("old", "impl", "expl0", "expl1")}
    return z, g, prof, mats, stw, stp


def test_update_wp_oracle():
    """The standard-form coupled (w, p) update with the l = 0 pressure restated in
    numpy against the reference's updateWP (Chebyshev, stress-free rows): new w,
    dw, ddw, p, dp and both equations' old, implicit and rotated explicit terms.
    The reference applies a precomputed inverse of the scaled 2N x 2N matrix, the
    oracle an LU solve; measured: w 2e-14, dw 1.1e-13, ddw 4e-13 (the derivatives
    amplify the solve's rounding), the rest <= 1.7e-14.  Bound 1e-12."""
    from oracle import implicit as oi

    z, g, prof, mats, stw, stp = _wp_case()
    o = oi.update_wp(g, mats, z["d3rMat"], prof, stw, stp, (z["wimp"], z["wimp_lin"], z["wexp"]),
                     z["hdif_V"], z["D1"], z["D2"], z["D3"], z["s_new"], float(z["BuoFac"]),
                     int(z["n_cheb_max"]), int(z["ktopv"]), int(z["kbotv"]))
    errs = {}
    for k in ("w", "dw", "ddw", "p", "dp"):
        errs[k] = rel_err(o[k], z[f"wp_{k}_new"])
    for f in ("w", "p"):
        for k in ("old", "impl", "expl1"):
            errs[f"{f}_{k}"] = rel_err(o[f"{f}_{k}"], z[f"wp_{f}_{k}_new"])
    print({k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < 1e-12, (k, v)


def test_wp_solve_operators():
    """The library's host builder of the coupled (w, p) solve operators (inverse of
    the scaled 2N x 2N matrix, Chebyshev truncation and DCT-I folded in), applied
    in numpy to the right-hand side, reproduces the reference's new w and p
    (degrees l >= 1; l = 0 takes the pressure operator)."""
    from types import SimpleNamespace

    from magic_b200 import implicit as I

    z, g, prof, mats, stw, stp = _wp_case()
    N = int(z["n_r_max"])
    sch = SimpleNamespace(n_r=N, chebyshev=True, n_cheb=int(z["n_cheb_max"]), rMat=z["rMat"],
                          drMat=z["drMat"], d2rMat=z["d2rMat"], d3rMat=z["d3rMat"],
                          rnorm=float(z["rnorm"]), boundary_fac=float(z["boundary_fac"]))
    w = I.cnab2_weights(1e-4, 1.3e-4)
    M = I.wp_solve_operators(sch, int(z["l_max"]), w[1], z["hdif_V"], prof, int(z["ktopv"]),
                             int(z["kbotv"]))
    rhs_of = lambda st: w[0] * st["old"] + w[2] * st["impl"] + w[3] * st["expl0"] \
        + w[4] * st["expl1"]
    rw, rp = rhs_of(stw), rhs_of(stp)
    rhs = np.zeros((rw.shape[0], 2 * N), dtype=np.complex128)
    rhs[:, 1:N - 1] = rw[:, 1:N - 1] + w[1] * float(z["BuoFac"]) * (
        z["rho0"] * z["rgrav"])[None, 1:N - 1] * z["s_new"][:, 1:N - 1]
    rhs[:, N + 1:2 * N - 1] = rp[:, 1:N - 1]
    x = np.stack([M[l] @ rhs[i] for i, l in enumerate(z["lm2l"])])
    x[z["lm2m"] == 0] = x[z["lm2m"] == 0].real
    P0 = I.p0_inverse(sch, z["beta"])
    p0_rhs = np.zeros(N)
    p0_rhs[1:] = z["rho0"][1:] * float(z["BuoFac"]) * z["rgrav"][1:] * z["s_new"][0, 1:].real \
        + stw["expl0"][0, 1:].real
    x[0, N:] = P0 @ p0_rhs
    assert rel_err(x[:, :N], z["wp_w_new"]) < 1e-12
    assert rel_err(x[:, N:], z["wp_p_new"]) < 1e-12


def test_wp_solve_operators_truncated():
    """With fewer Chebyshev modes than levels (n_cheb < n_r: boundary rows and the
    solution truncated, update_wp.py:309-313, 465-468) the library's folded
    operators reproduce the oracle's coupled solve on seeded right-hand sides."""
    from types import SimpleNamespace

    from magic_b200 import implicit as I
    from magic_b200.radial import cheb_polynomials
    from oracle import implicit as oi
    from oracle.td import dct1_matrix

    N, nc, l_max = 17, 14, 6
    T, dT, d2T, d3T = cheb_polynomials(N, 0.35, third=True)
    sch = SimpleNamespace(n_r=N, chebyshev=True, n_cheb=nc, rMat=T, drMat=dT, d2rMat=d2T,
                          d3rMat=d3T, rnorm=np.sqrt(2.0 / (N - 1)), boundary_fac=0.5)
    r = np.cos(np.pi * np.arange(N) / (N - 1)) * 0.5 + 1.5 / 1.3
    prof = dict(or1=1.0 / r, or2=1.0 / r ** 2, beta=-0.2 / r, dbeta=0.2 / r ** 2,
                visc=np.ones(N), dLvisc=np.zeros(N), rgrav=r, rho0=np.ones(N))
    hdif = np.ones(l_max + 1)
    wl0 = 0.6e-4
    M = I.wp_solve_operators(sch, l_max, wl0, hdif, prof, 1, 2)
    rng = np.random.default_rng(2)
    mats = (T, dT, d2T, sch.rnorm, sch.boundary_fac)
    C = dct1_matrix(N)
    for l in (1, 3, l_max):
        rhs = rng.standard_normal(2 * N) + 1j * rng.standard_normal(2 * N)
        rhs[[0, N - 1, N, 2 * N - 1]] = 0.0
        got = M[l] @ rhs
        dat = oi.wp_matrix(l, mats, d3T, prof, wl0, 1.0, nc, 1, 2)
        fr = 1.0 / np.abs(dat).max(axis=1)
        dat = fr[:, None] * dat
        fc = 1.0 / np.abs(dat).max(axis=0)
        y = fc * np.linalg.solve(dat * fc[None, :], fr * rhs)
        y[nc:N] = 0.0
        y[N + nc:] = 0.0
        ref = np.concatenate([C @ y[:N], C @ y[N:]])
        assert rel_err(got, ref) < 1e-11, (l, rel_err(got, ref))
