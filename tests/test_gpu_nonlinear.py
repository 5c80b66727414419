"""GPU parity of the grid-space nonlinear terms and the Courant check against the
reference golden vectors (FP64; pointwise formulas, tolerance 1e-13)."""

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu


def cu(x):
    return torch.as_tensor(np.ascontiguousarray(x)).cuda()


def npy(x):
    return x.detach().cpu().numpy()


def _plan(z):
    from magic_b200 import Plan

    p = Plan(int(z["l_max"]))
    assert (p.n_theta_max, p.n_phi_max) == (int(z["n_theta_max"]), int(z["n_phi_max"]))
    return p


def test_get_nl():
    z = load_golden("nl_bouss")
    p = _plan(z)
    names = ["vr", "vt", "vp", "cvr", "cvt", "cvp", "s", "br", "bt", "bp", "cbr", "cbt", "cbp", "xi"]
    res = p.get_nl([cu(z[k]) for k in names], cu(z["or2"]), cu(z["or4"]), float(z["LFfac"]))
    onames = ["Advr", "Advt", "Advp", "VSr", "VSt", "VSp", "VxBr", "VxBt", "VxBp", "VXir", "VXit",
              "VXip"]
    for k, v in zip(onames, res):
        assert rel_err(npy(v), z["out_" + k]) < 1e-13, k


def test_get_nl_reference_signature():
    import magic_b200
    from magic_b200.get_nl import get_nl

    z = load_golden("nl_bouss")
    magic_b200.configure({"l_max": int(z["l_max"]), "LFfac": float(z["LFfac"])})
    names = ["vr", "vt", "vp", "cvr", "cvt", "cvp", "s", "br", "bt", "bp", "cbr", "cbt", "cbp", "xi"]
    res = get_nl(*[cu(z[k]) for k in names], or4_3=cu(z["or4"]).reshape(-1, 1, 1),
                 or2_3=cu(z["or2"]).reshape(-1, 1, 1))
    assert rel_err(npy(res[0]), z["out_Advr"]) < 1e-13
    assert rel_err(npy(res[8]), z["out_VxBp"]) < 1e-13


def test_get_nl_anel():
    z = load_golden("nl_anel")
    p = _plan(z)
    names = ["vr", "vt", "vp", "dvrdr", "dvtdr", "dvpdr", "dvrdt", "dvrdp", "dvtdp", "dvpdp", "cvr",
             "s", "xi", "br", "bt", "bp", "cbr", "cbt", "cbp"]
    prof = {k: cu(z[k]) for k in ("r", "or1", "or2", "or4", "beta", "orho1", "otemp1", "visc",
                                  "lambda_")}
    res = p.get_nl_anel([cu(z[k]) for k in names], prof, float(z["LFfac"]),
                        float(z["ViscHeatFac"]), float(z["OhmLossFac"]))
    onames = ["Advr", "Advt", "Advp", "VSr", "VSt", "VSp", "VxBr", "VxBt", "VxBp", "VXir", "VXit",
              "VXip", "heat"]
    for k, v in zip(onames, res):
        assert rel_err(npy(v), z["out_" + k]) < 1e-13, k


def test_courant():
    z = load_golden("nl_bouss")
    p = _plan(z)
    prof = {k: cu(z[k]) for k in ("or2", "or4", "orho1", "orho2", "delxr2", "delxh2")}
    args = dict(courfac=float(z["courfac"]), alffac=float(z["alffac"]), LFfac=float(z["LFfac"]),
                opm=float(z["opm"]))
    v = [cu(z[k]) for k in ("vr", "vt", "vp")]
    b = [cu(z[k]) for k in ("br", "bt", "bp")]
    r, h = p.courant(*v, *b, prof, **args)
    assert rel_err(npy(r), z["cour_damp_r"]) < 1e-14 and rel_err(npy(h), z["cour_damp_h"]) < 1e-14
    r, h = p.courant(*v, None, None, None, prof, **args)
    assert rel_err(npy(r), z["cour_nomag_r"]) < 1e-14
    assert rel_err(npy(h), z["cour_nomag_h"]) < 1e-14
    r, h = p.courant(*v, *b, prof, damp=False, **args)
    np.testing.assert_allclose(npy(r), np.sqrt(z["delxr2"] / z["cour_nodamp_vr2"]), rtol=1e-14)
    np.testing.assert_allclose(npy(h), np.sqrt(z["delxh2"] / z["cour_nodamp_vh2"]), rtol=1e-14)
    # a resting fluid gives the 1e10 sentinel (courant.py:123-125)
    zero = torch.zeros_like(v[0])
    r, h = p.courant(zero, zero, zero, None, None, None, prof, **args)
    assert (npy(r) == 1e10).all() and (npy(h) == 1e10).all()
