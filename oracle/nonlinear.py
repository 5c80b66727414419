"""CPU oracle: grid-space nonlinear products and the Courant reduction.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Plain numpy, FP64.

The reference reads radial and theta profiles from module globals; here they
are explicit arguments.  Radial profiles are 1-D arrays over the levels of
the grids passed in, theta profiles are 1-D over the interleaved theta rows.

Restates ``get_nl.py:30-87`` (Boussinesq, curl-form advection),
``get_nl_anel.py:41-136`` (anelastic, u.grad u advection, viscous and Ohmic
heating) and ``courant.py:25-155``.
"""

import numpy as np


def _r3(a):
    return np.asarray(a, dtype=np.float64).reshape(-1, 1, 1)


def _t3(a):
    return np.asarray(a, dtype=np.float64).reshape(1, -1, 1)


def get_nl(vr, vt, vp, cvr, cvt, cvp, s, br, bt, bp, cbr, cbt, cbp, xi,
           or2, or4, ost2, LFfac):
    """Boussinesq products (``get_nl.py:57-87``).

    Returns (Advr, Advt, Advp, VSr, VSt, VSp, VxBr, VxBt, VxBp, VXir, VXit, VXip).
    """
    or2, or4, ost2 = _r3(or2), _r3(or4), _t3(ost2)
    LFr = LFfac * ost2 * (cbt * bp - cbp * bt)
    LFt = LFfac * or4 * (cbp * br - cbr * bp)
    LFp = LFfac * or4 * (cbr * bt - cbt * br)
    Advr = -ost2 * (cvt * vp - cvp * vt) + LFr
    Advt = -or4 * (cvp * vr - cvr * vp) + LFt
    Advp = -or4 * (cvr * vt - cvt * vr) + LFp
    VSr = vr * s
    VSt = or2 * vt * s
    VSp = or2 * vp * s
    VxBr = ost2 * (vt * bp - vp * bt)
    VxBt = or4 * (vp * br - vr * bp)
    VxBp = or4 * (vr * bt - vt * br)
    VXir = vr * xi
    VXit = or2 * vt * xi
    VXip = or2 * vp * xi
    return Advr, Advt, Advp, VSr, VSt, VSp, VxBr, VxBt, VxBp, VXir, VXit, VXip


def get_nl_anel(vr, vt, vp, dvrdr, dvtdr, dvpdr, dvrdt, dvrdp, dvtdp, dvpdp,
                cvr, s, xi, br, bt, bp, cbr, cbt, cbp,
                r, or1, or2, or4, beta, orho1, otemp1, visc, lambda_,
                ost2, cosn, LFfac, ViscHeatFac, OhmLossFac, l_mag=True):
    """Anelastic products with viscous/Ohmic heating (``get_nl_anel.py:63-136``).

    Returns the 12 arrays of ``get_nl`` followed by heatTerms.
    """
    r, or1, or2, or4 = _r3(r), _r3(or1), _r3(or2), _r3(or4)
    beta, orho1, otemp1 = _r3(beta), _r3(orho1), _r3(otemp1)
    visc, lam = _r3(visc), _r3(lambda_)
    ost2, cosn = _t3(ost2), _t3(cosn)
    LFr = LFfac * ost2 * (cbt * bp - cbp * bt)
    LFt = LFfac * or4 * (cbp * br - cbr * bp)
    LFp = LFfac * or4 * (cbr * bt - cbt * br)
    Advr = -or2 * orho1 * (vr * (dvrdr - (2.0 * or1 + beta) * vr)
                           + ost2 * (vt * (dvrdt - r * vt) + vp * (dvrdp - r * vp)))
    Advt = or4 * orho1 * (-vr * (dvtdr - beta * vt)
                          + vt * (cosn * vt + dvpdp + dvrdr)
                          + vp * (cosn * vp - dvtdp))
    Advp = or4 * orho1 * (-vr * (dvpdr - beta * vp) - vt * (dvtdp + cvr) - vp * dvpdp)
    Advr = Advr + LFr
    Advt = Advt + LFt
    Advp = Advp + LFp
    VSr = vr * s
    VSt = or2 * vt * s
    VSp = or2 * vp * s
    VxBr = orho1 * ost2 * (vt * bp - vp * bt)
    VxBt = orho1 * or4 * (vp * br - vr * bp)
    VxBp = orho1 * or4 * (vr * bt - vt * br)
    VXir = vr * xi
    VXit = or2 * vt * xi
    VXip = or2 * vp * xi
    prefac = ViscHeatFac * or4 * orho1 * otemp1 * visc
    beta_r = beta * r
    e_rr = dvrdr - (2.0 * or1 + beta) * vr
    e_tt = cosn * vt + dvpdp + dvrdr - or1 * vr
    e_pp = dvpdp + cosn * vt + or1 * vr
    e_tp = 2.0 * dvtdp + cvr - 2.0 * cosn * vp
    e_rt = r * dvtdr - (2.0 + beta_r) * vt + or1 * dvrdt
    e_rp = r * dvpdr - (2.0 + beta_r) * vp + or1 * dvrdp
    heat = prefac * (2.0 * e_rr * e_rr + 2.0 * e_tt * e_tt + 2.0 * e_pp * e_pp
                     + e_tp * e_tp + ost2 * (e_rt * e_rt + e_rp * e_rp)
                     - 2.0 * (1.0 / 3.0) * (beta * vr) ** 2)
    if l_mag and OhmLossFac != 0.0:
        heat = heat + OhmLossFac * lam * or2 * otemp1 * (
            or2 * cbr * cbr + ost2 * (cbt * cbt + cbp * cbp))
    return (Advr, Advt, Advp, VSr, VSt, VSp, VxBr, VxBt, VxBp,
            VXir, VXit, VXip, heat)


def courant_check(vr, vt, vp, br, bt, bp, courfac, alffac, or2, or4, orho1,
                  orho2, ost2, delxr2, delxh2, LFfac, opm, damp=True):
    """Per-level Courant steps (dtrkc, dthkc) (``courant.py:25-127``).

    ``br`` is None for the non-magnetic form.  ``damp`` selects the Alfven
    damping form (``courant.py:26-42``) or the undamped one (``:46-64``).
    """
    or2, or4, orho1, orho2 = _r3(or2), _r3(or4), _r3(orho1), _r3(orho2)
    ost2 = _t3(ost2)
    delxr2 = np.asarray(delxr2, dtype=np.float64)
    delxh2 = np.asarray(delxh2, dtype=np.float64)
    cf2 = courfac * courfac
    vflr2 = orho2 * vr * vr
    vflh2 = (vt * vt + vp * vp) * ost2 * orho2
    if br is not None:
        af2 = alffac * alffac
        valr = br * br * LFfac * orho1
        valh2 = (bt * bt + bp * bp) * LFfac * ost2 * orho1
        if damp:
            valri2 = ((0.5 * (1.0 + opm)) ** 2 / delxr2).reshape(-1, 1, 1)
            valhi2 = ((0.5 * (1.0 + opm)) ** 2 / delxh2).reshape(-1, 1, 1)
            valr2 = valr * valr / (valr + valri2)
            valh2m = valh2 * valh2 / (valh2 + valhi2)
        else:
            valr2 = valr
            valh2m = valh2
        vr2 = (or4 * (cf2 * vflr2 + af2 * valr2)).max(axis=(1, 2))
        vh2 = (or2 * (cf2 * vflh2 + af2 * valh2m)).max(axis=(1, 2))
    else:
        vr2 = (cf2 * or4 * vflr2).max(axis=(1, 2))
        vh2 = (cf2 * or2 * vflh2).max(axis=(1, 2))
    with np.errstate(divide="ignore", invalid="ignore"):
        dtr = np.where(vr2 > 0, np.sqrt(delxr2 / np.where(vr2 > 0, vr2, 1.0)), 1e10)
        dth = np.where(vh2 > 0, np.sqrt(delxh2 / np.where(vh2 > 0, vh2, 1.0)), 1e10)
    return dtr, dth


def dt_courant(dt, dtMax, dtrkc_min, dthkc_min):
    """Time-step hysteresis (``courant.py:130-155``): (changed, new_dt)."""
    dt_fac = 2.0
    dtMin = min(dtrkc_min, dthkc_min)
    dt_2 = min(0.5 * (1.0 / dt_fac + 1.0) * dtMin, dtMax)
    if dt > dtMax:
        return True, dtMax
    if dt > dtMin:
        return True, dt_2
    if dt_fac * dt < dtMin and dt < dtMax:
        return True, dt_2
    return False, dt
