"""CPU oracle: the nonlinear stage of one Boussinesq (and one anelastic) radial loop.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Plain numpy, FP64.

Restates ``step_time.py:931-1213`` steps 1-3 and 7 (the part the fused GPU
stage replaces): input assembly (``:980-1013``), batched inverse transforms,
``get_nl`` on all levels, forward transforms of the bulk levels 1..N-2
(``:1066-1124``) and the per-level Courant steps (``:1204-1212``).  Built
from the pinned pieces in ``oracle.sht`` and ``oracle.nonlinear``.
``nl_anel_stage`` restates ``radial_loop_anel`` (``step_time.py:1215-1475``)
from the same pieces.
"""

import numpy as np

from . import nonlinear as onl
from . import sht as osht


def nl_bouss_stage(g, f, prof, LFfac, courfac, alffac, opm, l_mag=True, l_chem=False,
                   damp=True):
    """``f``: dict of (lm_max, N) complex spectra w dw ddw z dz s [b db ddb aj dj] [xi].

    Returns (outputs dict of (lm_max, N) arrays with zero boundary columns,
    dtrkc, dthkc).
    """
    N = f["w"].shape[1]
    bulk = slice(1, N - 1)
    dLh = g.dLh[:, None]
    or2 = np.asarray(prof["or2"])[None, :]
    zeros = np.zeros((N, g.n_theta_max, g.n_phi_max))
    sc = osht.scal_to_spat(g, f["s"])
    xic = osht.scal_to_spat(g, f["xi"]) if l_chem else zeros
    if l_mag:
        br, bt, bp = osht.torpol_to_spat(g, dLh * f["b"], f["db"], f["aj"])
        cbr, cbt, cbp = osht.torpol_to_spat(g, dLh * f["aj"], f["dj"],
                                            or2 * dLh * f["b"] - f["ddb"])
    else:
        br = bt = bp = cbr = cbt = cbp = zeros
    vr, vt, vp = osht.torpol_to_spat(g, dLh * f["w"], f["dw"], f["z"])
    cvr, cvt, cvp = osht.torpol_to_spat(g, dLh * f["z"], f["dz"],
                                        or2 * dLh * f["w"] - f["ddw"])
    nl = onl.get_nl(vr, vt, vp, cvr, cvt, cvp, sc, br, bt, bp, cbr, cbt, cbp, xic,
                    prof["or2"], prof["or4"], g.O_sin_theta_E2_grid, LFfac)
    Advr, Advt, Advp, VSr, VSt, VSp, VxBr, VxBt, VxBp, VXir, VXit, VXip = nl
    out = {}

    def put(name, x):
        a = np.zeros((g.lm_max, N), dtype=np.complex128)
        a[:, bulk] = x
        out[name] = a

    put("Advr", osht.scal_to_SH(g, Advr[bulk]))
    put("VSr", osht.scal_to_SH(g, VSr[bulk]))
    s_, t_ = osht.spat_to_sphertor(g, Advt[bulk], Advp[bulk])
    put("Advt", s_)
    put("Advp", t_)
    put("VSt", osht.spat_to_sphertor(g, VSt[bulk], VSp[bulk])[0])
    if l_mag:
        put("VxBr", osht.scal_to_SH(g, VxBr[bulk]))
        s_, t_ = osht.spat_to_sphertor(g, VxBt[bulk], VxBp[bulk])
        put("VxBt", s_)
        put("VxBp", t_)
    if l_chem:
        put("VXir", osht.scal_to_SH(g, VXir[bulk]))
        put("VXit", osht.spat_to_sphertor(g, VXit[bulk], VXip[bulk])[0])
    dtr, dth = onl.courant_check(vr, vt, vp, br if l_mag else None, bt, bp, courfac, alffac,
                                 prof["or2"], prof["or4"], prof["orho1"], prof["orho2"],
                                 g.O_sin_theta_E2_grid, prof["delxr2"], prof["delxh2"], LFfac,
                                 opm, damp=damp)
    return out, dtr, dth


def bouss_profiles(N, radratio=0.35, l_max=16, seed=0):
    """Boussinesq radial profiles on N Chebyshev-Gauss-Lobatto radii.

    r_k = r_icb + (r_cmb - r_icb)(1 + cos(pi k/(N-1)))/2 (outer boundary first),
    or2 = 1/r^2, or4 = 1/r^4, orho = 1, delxr2/delxh2 as
    ``radial_functions.py:190-197``.
    """
    r_cmb = 1.0 / (1.0 - radratio)
    r_icb = r_cmb - 1.0
    k = np.arange(N)
    r = r_icb + (r_cmb - r_icb) * 0.5 * (1.0 + np.cos(np.pi * k / (N - 1)))
    dr = r[:-1] - r[1:]
    delxr2 = np.empty(N)
    delxr2[0] = dr[0] ** 2
    delxr2[-1] = dr[-1] ** 2
    delxr2[1:-1] = np.minimum(dr[:-1], dr[1:]) ** 2
    return dict(r=r, or2=1.0 / r ** 2, or4=1.0 / r ** 4, orho1=np.ones(N), orho2=np.ones(N),
                delxr2=delxr2, delxh2=r ** 2 / float(l_max * (l_max + 1)))


def nl_anel_stage(g, f, prof, LFfac, ViscHeatFac, OhmLossFac, courfac, alffac, opm,
                  l_mag=True, l_chem=False, damp=True):
    """Nonlinear part of ``radial_loop_anel`` (``step_time.py:1215-1475``).

    ``f``: dict of (lm_max, N) spectra w dw ddw z dz s [xi] [b db ddb aj dj].
    Velocity, its radial/horizontal derivatives and cvr are synthesised on the
    bulk levels only and are zero on the two boundaries (``:1266-1316``);
    s, xi and the magnetic field on all levels (``:1233-1262``).  Products by
    ``get_nl_anel`` (``:1319-1326``), forward transforms of the bulk levels
    (``:1329-1391``), Courant steps from the zero-boundary velocity
    (``:1466-1474``).  Returns (outputs dict with zero boundary columns:
    Advr Advt Advp VSr VSt [VxBr VxBt VxBp] [VXir VXit] heat, dtrkc, dthkc).
    """
    N = f["w"].shape[1]
    bulk = slice(1, N - 1)
    dLh = g.dLh[:, None]
    or2 = np.asarray(prof["or2"])[None, :]
    shape = (N, g.n_theta_max, g.n_phi_max)
    zeros = np.zeros(shape)
    sc = osht.scal_to_spat(g, f["s"])
    xic = osht.scal_to_spat(g, f["xi"]) if l_chem else zeros
    if l_mag:
        br, bt, bp = osht.torpol_to_spat(g, dLh * f["b"], f["db"], f["aj"])
        cbr, cbt, cbp = osht.torpol_to_spat(g, dLh * f["aj"], f["dj"],
                                            or2 * dLh * f["b"] - f["ddb"])
    else:
        br = bt = bp = cbr = cbt = cbp = zeros

    def bulk_only(grids):
        out = []
        for x in grids:
            a = np.zeros(shape)
            a[bulk] = x
            out.append(a)
        return out

    w, dw, ddw, z, dz = (f[k][:, bulk] for k in ("w", "dw", "ddw", "z", "dz"))
    d = dLh
    vr, vt, vp = bulk_only(osht.torpol_to_spat(g, d * w, dw, z))
    dvrdr, dvtdr, dvpdr = bulk_only(osht.torpol_to_spat(g, d * dw, ddw, dz))
    (cvr,) = bulk_only([osht.pol_to_curlr_spat(g, z)])
    dvrdt, dvrdp = bulk_only(osht.pol_to_grad_spat(g, w))
    dvtdp, dvpdp = bulk_only(osht.torpol_to_dphspat(g, dw, z))
    nl = onl.get_nl_anel(vr, vt, vp, dvrdr, dvtdr, dvpdr, dvrdt, dvrdp, dvtdp, dvpdp, cvr, sc,
                         xic, br, bt, bp, cbr, cbt, cbp, prof["r"], prof["or1"], prof["or2"],
                         prof["or4"], prof["beta"], prof["orho1"], prof["otemp1"],
                         prof["visc"], prof["lambda_"], g.O_sin_theta_E2_grid,
                         g.cosn_theta_E2_grid, LFfac, ViscHeatFac, OhmLossFac, l_mag)
    Advr, Advt, Advp, VSr, VSt, VSp, VxBr, VxBt, VxBp, VXir, VXit, VXip, heat = nl
    out = {}

    def put(name, x):
        a = np.zeros((g.lm_max, N), dtype=np.complex128)
        a[:, bulk] = x
        out[name] = a

    put("Advr", osht.scal_to_SH(g, Advr[bulk]))
    put("VSr", osht.scal_to_SH(g, VSr[bulk]))
    s_, t_ = osht.spat_to_sphertor(g, Advt[bulk], Advp[bulk])
    put("Advt", s_)
    put("Advp", t_)
    put("VSt", osht.spat_to_sphertor(g, VSt[bulk], VSp[bulk])[0])
    if l_mag:
        put("VxBr", osht.scal_to_SH(g, VxBr[bulk]))
        s_, t_ = osht.spat_to_sphertor(g, VxBt[bulk], VxBp[bulk])
        put("VxBt", s_)
        put("VxBp", t_)
    if l_chem:
        put("VXir", osht.scal_to_SH(g, VXir[bulk]))
        put("VXit", osht.spat_to_sphertor(g, VXit[bulk], VXip[bulk])[0])
    put("heat", osht.scal_to_SH(g, heat[bulk]))
    dtr, dth = onl.courant_check(vr, vt, vp, br if l_mag else None, bt, bp, courfac, alffac,
                                 prof["or2"], prof["or4"], prof["orho1"], prof["orho2"],
                                 g.O_sin_theta_E2_grid, prof["delxr2"], prof["delxh2"], LFfac,
                                 opm, damp=damp)
    return out, dtr, dth


def anel_profiles(N, radratio=0.35, l_max=16, strat=5.0, polind=2.0):
    """Anelastic radial profiles on N Chebyshev-Gauss-Lobatto radii: a
    polytrope of index ``polind`` with ``strat`` density scale heights
    (temp0 = 1 + c (r_cmb / r - 1) normalised to 1 at r_cmb, rho0 = temp0^n,
    beta = d ln rho0 / dr, otemp1 = 1/temp0, orho1 = 1/rho0, orho2 = orho1^2),
    unit viscosity and magnetic diffusivity, delxr2/delxh2 as
    ``bouss_profiles``.  Test inputs, not the reference's radial functions."""
    p = bouss_profiles(N, radratio, l_max)
    r = p["r"]
    r_cmb = 1.0 / (1.0 - radratio)
    r_icb = r_cmb - 1.0
    c = (np.exp(strat / polind) - 1.0) / (r_cmb / r_icb - 1.0)
    temp0 = 1.0 + c * (r_cmb / r - 1.0)
    rho0 = temp0 ** polind
    dtemp0 = -c * r_cmb / r ** 2
    beta = polind * dtemp0 / temp0
    p.update(or1=1.0 / r, beta=beta, otemp1=1.0 / temp0, orho1=1.0 / rho0, orho2=1.0 / rho0 ** 2,
             visc=np.ones(N), lambda_=np.ones(N))
    return p
