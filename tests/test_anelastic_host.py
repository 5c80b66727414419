"""Host-side pieces of the anelastic time step against values the reference
computed (tests/golden/step_anel.npz, td_fd_anel.npz): the polytropic
background (magic_torch/radial_functions.py:70-165) on Chebyshev and FD radii,
the viscous-heating factor, and the angular-momentum correction constants
(pre_calculations.py:94-98, update_z.py:57-64) with this package's radial
rule.  No GPU."""

import json

import numpy as np

from conftest import load_golden


def _bg(z, cfg):
    from magic_b200.profiles import polytropic_background

    return polytropic_background(z["r"], 0.35, cfg["strat"], cfg["polind"], cfg["g0"], cfg["g1"],
                                 cfg["g2"], cfg["pr"], cfg["ra"], cfg["ek"], cfg["prmag"])


def test_background_matches_reference_on_chebyshev_levels():
    z = load_golden("step_anel")
    cfg = json.loads(str(z["cfg"]))
    bg = _bg(z, cfg)
    for k in ("rho0", "beta", "dbeta", "rgrav", "dLtemp0", "otemp1"):
        e = np.abs(bg[k] - z[k]).max() / np.abs(z[k]).max()
        assert e < 1e-14, (k, e)
    assert abs(bg["ViscHeatFac"] - float(z["ViscHeatFac"])) <= 1e-15 * float(z["ViscHeatFac"])


def test_background_matches_reference_on_fd_levels():
    z = load_golden("td_fd_anel")
    cfg = dict(strat=5.0, polind=2.0, g0=0.0, g1=0.0, g2=1.0, pr=1.0, ra=3e6, ek=1e-4, prmag=5.0)
    bg = _bg(z, cfg)
    for k in ("rho0", "beta", "dbeta", "ddbeta", "rgrav", "dLtemp0", "orho1"):
        e = np.abs(bg[k] - z[k]).max() / np.abs(z[k]).max()
        assert e < 1e-14, (k, e)


def test_angular_momentum_constants():
    """c_moi_oc = 8/3 pi int r^4 rho0 dr with the Clenshaw-Curtis rule of the
    Chebyshev levels equals the reference's; the correction profiles are the
    radial derivatives of rho0 r^2 (am_dz = d(am_z)/dr - ... as update_z.py
    states them: rho0' = beta rho0)."""
    from magic_b200.implicit import am_profiles
    from magic_b200.radial import clenshaw_curtis_weights

    z = load_golden("step_anel")
    N = int(z["n_r_max"])
    rint = clenshaw_curtis_weights(N, 0.35, np.sqrt(2.0 / (N - 1)), 0.5)
    assert np.abs(rint - z["rint_w"]).max() < 1e-14 * np.abs(z["rint_w"]).max()
    p = am_profiles(z["r"], z["rho0"], z["beta"], z["dbeta"], rint)
    assert abs(p["c_moi_oc"] - float(z["c_moi_oc"])) < 1e-13 * float(z["c_moi_oc"])
    r, rho0, beta, dbeta = z["r"], z["rho0"], z["beta"], z["dbeta"]
    # d(rho0 r^2)/dr = rho0 (2 r + beta r^2); d2/dr2 = rho0 (2 + 4 beta r + (dbeta + beta^2) r^2)
    assert np.allclose(p["am_z"], rho0 * r * r, rtol=1e-15)
    assert np.allclose(p["am_dz"], rho0 * (2 * r + beta * r * r), rtol=1e-15)
    assert np.allclose(p["am_d2z"], rho0 * (2 + 4 * beta * r + (dbeta + beta ** 2) * r * r),
                       rtol=1e-15)
