"""Generate golden input/output vectors by running the reference itself.

Usage (in a container where the reference source is available):

    python tests/golden/make_golden.py --ref /root/reference/src

Each configuration runs in its own subprocess because the reference reads its
parameters at import time (one process = one configuration).  The reference
runs on the CPU in FP64 with TorchDynamo disabled (its ``@torch.compile``
functions then run eagerly, which the reference documents as bit-identical).

Outputs ``tests/golden/<name>.npz``.  Inputs are seeded numpy draws; the
fixtures hold both inputs and reference outputs so the tests never need the
reference at run time.
"""

import argparse
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

SHT_CONFIGS = {
    # name: (configure dict, batch columns, store tables)
    "sht_l16": ({"l_max": 16, "minc": 1, "n_r_max": 5}, 3, True),
    "sht_l32m4": ({"l_max": 32, "minc": 4, "n_r_max": 5}, 3, True),
    "sht_l20": ({"l_max": 20, "minc": 1, "n_r_max": 5}, 2, True),
    "sht_l31m2": ({"l_max": 31, "minc": 2, "n_r_max": 5}, 2, True),
    "sht_l64": ({"l_max": 64, "minc": 1, "n_r_max": 5}, 1, False),
}

NL_CONFIGS = {
    "nl_bouss": {"l_max": 8, "minc": 1, "n_r_max": 4, "mode": 0},
    "nl_anel": {"l_max": 8, "minc": 1, "n_r_max": 5, "strat": 5.0, "polind": 2.0,
                "g0": 0.0, "g1": 0.0, "g2": 1.0, "mode": 0, "ek": 1e-4, "ra": 3e6},
}


# whole CNAB2 steps of the Boussinesq MHD dynamo (insulating inner core, fixed
# entropy, no-slip): fourth-order FD with the double-curl form, and Chebyshev
# levels with the standard form
STEP_CONFIGS = {
    # Chebyshev levels, standard (w, p) form, minc 4
    "step_cheb": {"l_max": 32, "minc": 4, "n_r_max": 33, "ek": 1e-3, "ra": 1e5, "pr": 1.0,
                  "prmag": 5.0, "dtmax": 5e-6, "mode": 0},
    "step_fd": {"l_max": 12, "minc": 1, "n_r_max": 13, "radial_scheme": "FD", "fd_order": 4,
                "fd_order_bound": 2, "ek": 1e-3, "ra": 1e5, "pr": 1.0, "prmag": 5.0,
                "dtmax": 1e-4, "mode": 0},
    # anelastic convection without magnetic field (the reference's anelastic
    # benchmark setup, configs/hydro_bench_anel_modal.yaml, at a small size):
    # polytropic background with 5 density scale heights, index 2, gravity
    # ~ 1/r^2, stress-free boundaries with both angular-momentum corrections,
    # Chebyshev levels, standard (w, p) form
    "step_anel": {"l_max": 16, "minc": 1, "n_r_max": 17, "strat": 5.0, "polind": 2.0,
                  "g0": 0.0, "g1": 0.0, "g2": 1.0, "mode": 1, "ek": 1e-3, "ra": 1.48638035e5,
                  "pr": 1.0, "prmag": 5.0, "ktopv": 1, "kbotv": 1, "l_correct_AMz": True,
                  "l_correct_AMe": True, "dtmax": 1e-4},
}

# 500 CNAB2 steps of the Boussinesq MHD dynamo at the sizes of the CPU-runnable
# shell case (l_max 32, minc 4, 33 levels, Ek 1e-3, Ra 1e5, Pr 1, Pm 5, dt 1e-4,
# the reference's initial fields: l = m = 4 entropy mode of amplitude 0.1 and
# its dipolar poloidal field, init_b1 = 3, amp_b1 = 5) with seeded Gaussian
# noise of amplitude 1e-5 on the entropy; on its 33 Chebyshev levels (standard
# (w, p) form) and on 33 fourth-order FD levels (double-curl form).
RUN_CONFIGS = {
    # the shell case itself: 33 Chebyshev levels, standard (w, p) form
    "run_cheb_l32m4": ({"l_max": 32, "minc": 4, "n_r_max": 33, "ek": 1e-3, "ra": 1e5,
                        "pr": 1.0, "prmag": 5.0, "dtmax": 1e-4, "mode": 0}, 500, 1e-5),
    "run_fd_l32m4": ({"l_max": 32, "minc": 4, "n_r_max": 33, "radial_scheme": "FD",
                      "fd_order": 4, "fd_order_bound": 2, "ek": 1e-3, "ra": 1e5, "pr": 1.0,
                      "prmag": 5.0, "dtmax": 1e-4, "mode": 0}, 500, 1e-5),
    # 100 steps of the anelastic setup of step_anel at l_max 32 on 33 Chebyshev
    # levels from the benchmark's l = m = 19 entropy mode (init_s1 1919, amplitude
    # 0.01) plus seeded noise of 1e-3 on the entropy
    "run_anel_l32": ({"l_max": 32, "minc": 1, "n_r_max": 33, "strat": 5.0, "polind": 2.0,
                      "g0": 0.0, "g1": 0.0, "g2": 1.0, "mode": 1, "ek": 1e-3,
                      "ra": 1.48638035e5, "pr": 1.0, "prmag": 5.0, "ktopv": 1, "kbotv": 1,
                      "l_correct_AMz": True, "l_correct_AMe": True, "init_s1": 1919,
                      "amp_s1": 0.01, "dtmax": 1e-4}, 100, 1e-3),
}

# CNAB2 steps with the Courant control of dt (courant.py:130-155; one_step
# changes dt and rebuilds the matrices when the limit requires): the shell case
# on Chebyshev levels with dtmax 1e-4 and seeded perturbations of s, w and z of
# 1e-3, where the first step already cuts dt
ADAPT_CONFIGS = {
    "adapt_cheb": ({"l_max": 32, "minc": 4, "n_r_max": 33, "ek": 1e-3, "ra": 1e5, "pr": 1.0,
                    "prmag": 5.0, "dtmax": 1e-4, "mode": 0}, 30),
}

# energies of seeded spectra (output.py:101-180) and the radial rule
ENERGY_CONFIGS = {
    "energy_cheb": {"l_max": 8, "minc": 2, "n_r_max": 11, "prmag": 5.0, "ek": 1e-3},
    "energy_fd": {"l_max": 12, "minc": 1, "n_r_max": 12, "radial_scheme": "FD", "fd_order": 4,
                  "fd_order_bound": 2, "strat": 2.0, "polind": 2.0, "g0": 0.0, "g1": 0.0,
                  "g2": 1.0, "mode": 0, "ek": 1e-4, "ra": 3e6},
}


def _spec(rng, lm_max, l_of_lm, B, decay=1.0):
    """Random complex spectrum with |c| ~ (l+1)^-decay."""
    amp = (l_of_lm.astype(np.float64) + 1.0) ** (-decay)
    x = (rng.standard_normal((lm_max, B)) + 1j * rng.standard_normal((lm_max, B)))
    return x * amp[:, None]


def worker_sht(name, ref):
    cfg, B, tables = SHT_CONFIGS[name]
    cfg = dict(cfg, device="cpu", use_shtns=False)
    sys.path.insert(0, ref)
    from magic_torch.config import configure
    configure(cfg)
    import torch
    from magic_torch import params, sht, plms, horizontal_data as hd, blocking
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))
    n = lambda x: x.detach().cpu().numpy()
    rng = np.random.default_rng(1234)
    lm, nt, npp = params.lm_max, params.n_theta_max, params.n_phi_max
    l_of = n(blocking.st_lm2l)
    out = dict(l_max=params.l_max, minc=params.minc, lm_max=lm,
               n_theta_max=nt, n_phi_max=npp, n_m_max=params.n_m_max)
    # Slm keeps a nonzero imaginary part at m=0: irfft must drop it.
    Slm = _spec(rng, lm, l_of, B)
    Q, S, T = (_spec(rng, lm, l_of, B) for _ in range(3))
    grid = rng.standard_normal((B, nt, npp))
    vt = rng.standard_normal((B, nt, npp))
    vp = rng.standard_normal((B, nt, npp))
    or2 = 1.0 + rng.random(B)
    Bl, ddB, J, dJ = (_spec(rng, lm, l_of, B) for _ in range(4))
    out.update(Slm=Slm, Q=Q, S=S, T=T, grid=grid, vt=vt, vp=vp, or2=or2,
               Bl=Bl, ddB=ddB, J=J, dJ=dJ)
    out["scal_to_spat"] = n(sht.scal_to_spat(t(Slm)))
    out["scal_to_spat_1d"] = n(sht.scal_to_spat(t(Slm[:, 0].copy())))
    out["scal_to_SH"] = n(sht.scal_to_SH(t(grid)))
    out["scal_to_SH_1d"] = n(sht.scal_to_SH(t(grid[0].copy())))
    br, bt, bp = sht.torpol_to_spat(t(Q), t(S), t(T))
    out.update(torpol_br=n(br), torpol_bt=n(bt), torpol_bp=n(bp))
    br1, bt1, bp1 = sht.torpol_to_spat(t(Q[:, 0].copy()), t(S[:, 0].copy()), t(T[:, 0].copy()))
    out.update(torpol1_br=n(br1), torpol1_bt=n(bt1), torpol1_bp=n(bp1))
    s_, t_ = sht.spat_to_sphertor(t(vt), t(vp))
    out.update(sphertor_S=n(s_), sphertor_T=n(t_))
    s1, t1 = sht.spat_to_sphertor(t(vt[0].copy()), t(vp[0].copy()))
    out.update(sphertor1_S=n(s1), sphertor1_T=n(t1))
    gt, gp = sht.scal_to_grad_spat(t(Slm))
    out.update(grad_t=n(gt), grad_p=n(gp))
    out["curlr"] = n(sht.pol_to_curlr_spat(t(Q)))
    pg_t, pg_p = sht.pol_to_grad_spat(t(S))
    out.update(polgrad_t=n(pg_t), polgrad_p=n(pg_p))
    dt_, dp_ = sht.torpol_to_dphspat(t(S[:, 0].copy()), t(T[:, 0].copy()))
    out.update(dph_t=n(dt_), dph_p=n(dp_))
    cr, ct, cp = sht.torpol_to_curl_spat(t(or2), t(Bl), t(ddB), t(J), t(dJ))
    out.update(curl_r=n(cr), curl_t=n(ct), curl_p=n(cp))
    st_t, st_p = sht.sphtor_to_spat(t(S[:, 0].copy()), t(T[:, 0].copy()))
    out.update(sphtor_t=n(st_t), sphtor_p=n(st_p))
    q_, s2, t2 = sht.spat_to_qst(t(grid[0].copy()), t(vt[0].copy()), t(vp[0].copy()))
    out.update(qst_q=n(q_), qst_s=n(s2), qst_t=n(t2))
    e10 = np.zeros(lm, dtype=np.complex128)
    e10[1] = 1.0
    out["y10"] = n(sht.scal_to_spat(t(e10)))
    if tables:
        out.update(theta_ord=n(hd.theta_ord), gauss=n(hd.gauss), Plm=n(plms.Plm),
                   dPlm=n(plms.dPlm), wPlm=n(plms.wPlm), wdPlm=n(plms.wdPlm),
                   O_sin_theta_E2_grid=n(hd.O_sin_theta_E2_grid),
                   cosn_theta_E2_grid=n(hd.cosn_theta_E2_grid))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def worker_nl(name, ref):
    cfg = dict(NL_CONFIGS[name], device="cpu", use_shtns=False)
    sys.path.insert(0, ref)
    from magic_torch.config import configure
    configure(cfg)
    import torch
    from magic_torch import params, radial_functions as rf, horizontal_data as hd
    from magic_torch import pre_calculations as pc, courant
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))
    n = lambda x: x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)
    rng = np.random.default_rng(99)
    N, nt, npp = params.n_r_max, params.n_theta_max, params.n_phi_max
    out = dict(n_r_max=N, n_theta_max=nt, n_phi_max=npp, l_max=params.l_max,
               or1=n(rf.or1), or2=n(rf.or2), or4=n(rf.or4), r=n(rf.r) if hasattr(rf, "r") else None,
               orho1=n(rf.orho1), orho2=n(rf.orho2), otemp1=n(rf.otemp1),
               beta=n(rf.beta), visc=n(rf.visc), lambda_=n(rf.lambda_),
               delxr2=n(rf.delxr2), delxh2=n(rf.delxh2),
               ViscHeatFac=float(rf.ViscHeatFac), OhmLossFac=float(rf.OhmLossFac),
               LFfac=float(pc.LFfac), opm=float(pc.opm),
               ost2=n(hd.O_sin_theta_E2_grid), cosn=n(hd.cosn_theta_E2_grid))
    from magic_torch.radial_scheme import r as r_grid
    out["r"] = n(r_grid)
    g = lambda: rng.standard_normal((N, nt, npp))
    if name == "nl_bouss":
        from magic_torch.get_nl import get_nl
        names = ["vr", "vt", "vp", "cvr", "cvt", "cvp", "s", "br", "bt", "bp",
                 "cbr", "cbt", "cbp", "xi"]
        ins = {k: g() for k in names}
        res = get_nl(*[t(ins[k]) for k in names])
        onames = ["Advr", "Advt", "Advp", "VSr", "VSt", "VSp", "VxBr", "VxBt", "VxBp",
                  "VXir", "VXit", "VXip"]
        out.update(ins)
        out.update({"out_" + k: n(v) for k, v in zip(onames, res)})
        # Courant: damped magnetic (default), undamped, and non-magnetic forms.
        courfac, alffac = 2.5, 1.0
        out.update(courfac=courfac, alffac=alffac)
        d1, d2 = courant.courant_check(t(ins["vr"]), t(ins["vt"]), t(ins["vp"]),
                                       t(ins["br"]), t(ins["bt"]), t(ins["bp"]),
                                       courfac=courfac, alffac=alffac)
        out.update(cour_damp_r=n(d1), cour_damp_h=n(d2))
        d1, d2 = courant.courant_check(t(ins["vr"]), t(ins["vt"]), t(ins["vp"]),
                                       courfac=courfac, alffac=alffac)
        out.update(cour_nomag_r=n(d1), cour_nomag_h=n(d2))
        vr2, vh2 = courant._courant_mag_nodamp(
            t(ins["vr"]), t(ins["vt"]), t(ins["vp"]), t(ins["br"]), t(ins["bt"]),
            t(ins["bp"]), courfac ** 2, alffac ** 2)
        out.update(cour_nodamp_vr2=n(vr2), cour_nodamp_vh2=n(vh2))
        cases = [(1e-4, 1e-4, 1e-3, 2e-3), (2e-4, 1e-4, 1e-5, 3e-5),
                 (1e-6, 1e-4, 1e-3, 1e-3), (1e-5, 1e-4, 3e-5, 1e-4)]
        res = [courant.dt_courant(*c) for c in cases]
        out["dtc_cases"] = np.array(cases)
        out["dtc_changed"] = np.array([r_[0] for r_ in res])
        out["dtc_new"] = np.array([r_[1] for r_ in res])
    else:
        from magic_torch.get_nl_anel import get_nl_anel
        names = ["vr", "vt", "vp", "dvrdr", "dvtdr", "dvpdr", "dvrdt", "dvrdp",
                 "dvtdp", "dvpdp", "cvr", "s", "xi", "br", "bt", "bp", "cbr", "cbt", "cbp"]
        ins = {k: g() for k in names}
        res = get_nl_anel(*[t(ins[k]) for k in names])
        onames = ["Advr", "Advt", "Advp", "VSr", "VSt", "VSp", "VxBr", "VxBt", "VxBp",
                  "VXir", "VXit", "VXip", "heat"]
        out.update(ins)
        out.update({"out_" + k: n(v) for k, v in zip(onames, res)})
    out = {k: v for k, v in out.items() if v is not None}
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


TD_CONFIGS = {
    # spectral explicit terms (get_td + finish_exp), radial derivatives, DCT-I
    "td_cheb": {"l_max": 8, "minc": 1, "n_r_max": 9, "mode": 0, "ktopv": 1, "kbotv": 1},
    "td_fd_anel": {"l_max": 16, "minc": 2, "n_r_max": 12, "radial_scheme": "FD",
                   "fd_order": 4, "fd_order_bound": 2, "strat": 5.0, "polind": 2.0,
                   "g0": 0.0, "g1": 0.0, "g2": 1.0, "mode": 0, "ek": 1e-4, "ra": 3e6},
}


def worker_td(name, ref):
    cfg = dict(TD_CONFIGS[name], device="cpu", use_shtns=False)
    sys.path.insert(0, ref)
    from magic_torch.config import configure
    configure(cfg)
    import torch
    from magic_torch import params, blocking, radial_functions as rf, pre_calculations as pc
    from magic_torch import get_td as gt, radial_derivatives as rd
    from magic_torch.radial_scheme import r as r_grid
    from magic_torch.cosine_transform import costf
    from magic_torch.update_s import finish_exp_entropy
    from magic_torch.update_wp import finish_exp_pol
    from magic_torch.update_b import finish_exp_mag
    from magic_torch.update_xi import finish_exp_comp
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))
    # copies: updateS later overwrites its time arrays in place
    n = lambda x: x.detach().cpu().numpy().copy()
    rng = np.random.default_rng(321)
    N, lm = params.n_r_max, params.lm_max
    l_of = n(blocking.st_lm2l)
    out = dict(n_r_max=N, l_max=params.l_max, minc=params.minc, lm_max=lm,
               l_anel=int(bool(params.l_anel)), l_double_curl=int(bool(params.l_double_curl)),
               r=n(r_grid), or1=n(rf.or1), or2=n(rf.or2), or4=n(rf.or4), orho1=n(rf.orho1),
               beta=n(rf.beta), CorFac=float(pc.CorFac), lm2l=l_of, lm2m=n(blocking.st_lm2m),
               D1=n(rd._D1_real), D2=n(rd._D2_real))
    names = ["Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt", "VxBp", "VXir", "VXit",
             "w", "dw", "ddw", "z", "dz", "f"]
    ins = {k: _spec(rng, lm, l_of, N) for k in names}
    out.update({"in_" + k: v for k, v in ins.items()})
    T = {k: t(v) for k, v in ins.items()}
    out["dwdt"] = n(gt.get_dwdt(T["Advr"], T["dw"], T["z"]))
    dwdt_dc, dVxVh = gt.get_dwdt_double_curl(T["Advr"], T["Advt"], T["w"], T["dw"], T["ddw"],
                                             T["z"], T["dz"])
    out["dwdt_dc"] = n(dwdt_dc)
    out["dVxVh"] = n(dVxVh)
    out["dwdt_dc_fin"] = n(finish_exp_pol(dwdt_dc.clone(), dVxVh))
    out["dzdt"] = n(gt.get_dzdt(T["Advp"], T["w"], T["dw"], T["z"]))
    out["dpdt"] = n(gt.get_dpdt(T["Advt"], T["w"], T["dw"], T["z"]))
    ds, dVSr = gt.get_dsdt(T["VSt"], T["VSr"])
    out["dsdt_part"] = n(ds)
    out["dsdt"] = n(finish_exp_entropy(ds.clone(), dVSr))
    dx, dVXir = gt.get_dxidt(T["VXit"], T["VXir"])
    out["dxidt"] = n(finish_exp_comp(dx.clone(), dVXir))
    db, dj, dVxBh = gt.get_dbdt(T["VxBr"], T["VxBt"], T["VxBp"])
    out["dbdt"] = n(db)
    out["djdt_part"] = n(dj)
    out["djdt"] = n(finish_exp_mag(dj.clone(), dVxBh))
    out["dr_f"] = n(rd.get_dr(T["f"]))
    d1, d2 = rd.get_ddr(T["f"])
    out["ddr_f1"], out["ddr_f2"] = n(d1), n(d2)
    out["costf_f"] = n(costf(T["f"]))
    # one implicit entropy update (magic_torch/update_s.py:67-271) with CNAB2
    # weights from two different time steps
    from magic_torch.time_scheme import tscheme
    from magic_torch import update_s as us, dt_fields as dtf, horizontal_data as hd
    from magic_torch import radial_functions as rf2
    tscheme.dt[0] = 1e-4
    tscheme.dt[1] = 1.3e-4
    tscheme.set_weights()
    us.build_s_matrices(tscheme.wimp_lin[0].item())
    ta = dtf.TimeArray(tscheme.nold, tscheme.nexp, tscheme.nimp)
    ta.old[:, :, 0] = t(_spec(rng, lm, l_of, N))
    ta.impl[:, :, 0] = t(_spec(rng, lm, l_of, N))
    ta.expl[:, :, 0] = t(_spec(rng, lm, l_of, N))
    ta.expl[:, :, 1] = t(_spec(rng, lm, l_of, N))
    out.update(s_old=n(ta.old[:, :, 0]), s_impl=n(ta.impl[:, :, 0]),
               s_expl0=n(ta.expl[:, :, 0]), s_expl1=n(ta.expl[:, :, 1]),
               wimp=n(tscheme.wimp), wimp_lin=n(tscheme.wimp_lin), wexp=n(tscheme.wexp),
               opr=float(pc.opr), hdif_S=n(hd.hdif_S), kappa=n(rf2.kappa),
               dLtemp0=n(rf2.dLtemp0), dLkappa=n(rf2.dLkappa), bots=n(us._bots),
               tops=n(us._tops), n_cheb_max=int(params.n_cheb_max))
    from magic_torch import radial_scheme as rs
    out.update(rMat=n(rs.rMat), drMat=n(rs.drMat), d2rMat=n(rs.d2rMat),
               rnorm=float(rs.rnorm), boundary_fac=float(rs.boundary_fac),
               chebyshev=int(params.radial_scheme != "FD"))
    s_new = torch.zeros(lm, N, dtype=torch.complex128)
    ds_new = torch.zeros_like(s_new)
    us.updateS(s_new, ds_new, ta, tscheme)
    out.update(s_new=n(s_new), ds_new=n(ds_new), s_impl_new=n(ta.impl[:, :, 0]),
               s_old_new=n(ta.old[:, :, 0]), s_expl1_new=n(ta.expl[:, :, 1]))
    # one implicit toroidal-velocity update (magic_torch/update_z.py:89-505)
    from magic_torch import update_z as uz
    uz.build_z_matrices(tscheme.wimp_lin[0].item())
    tz = dtf.TimeArray(tscheme.nold, tscheme.nexp, tscheme.nimp)
    for k, arr in (("old", tz.old), ("impl", tz.impl), ("expl0", tz.expl), ("expl1", tz.expl)):
        v = _spec(rng, lm, l_of, N)
        arr[:, :, 1 if k == "expl1" else 0] = t(v)
        out["z_" + k] = v
    out.update(visc=n(rf2.visc), dLvisc=n(rf2.dLvisc), dbeta=n(rf2.dbeta),
               hdif_V=n(hd.hdif_V), ktopv=int(params.ktopv), kbotv=int(params.kbotv),
               fd_order=int(getattr(params, "fd_order", 2)))
    z_new = torch.zeros(lm, N, dtype=torch.complex128)
    dz_new = torch.zeros_like(z_new)
    uz.updateZ(z_new, dz_new, tz, tscheme)
    out.update(z_new=n(z_new), dz_new=n(dz_new), z_impl_new=n(tz.impl[:, :, 0]),
               z_old_new=n(tz.old[:, :, 0]), z_expl1_new=n(tz.expl[:, :, 1]))
    # one implicit magnetic update, insulating inner core (update_b.py:98-635)
    from magic_torch import update_b as ub
    ub.build_b_matrices(tscheme.wimp_lin[0].item())
    tb = dtf.TimeArray(tscheme.nold, tscheme.nexp, tscheme.nimp)
    tj = dtf.TimeArray(tscheme.nold, tscheme.nexp, tscheme.nimp)
    for f, ta_ in (("b", tb), ("j", tj)):
        for k in ("old", "impl", "expl0", "expl1"):
            v = _spec(rng, lm, l_of, N)
            (ta_.old if k == "old" else ta_.impl if k == "impl" else ta_.expl)[
                :, :, 1 if k == "expl1" else 0] = t(v)
            out[f + "_" + k] = v
    out.update(opm=float(pc.opm), lambda_=n(rf2.lambda_), dLlambda=n(rf2.dLlambda),
               hdif_B=n(hd.hdif_B))
    bj = [torch.zeros(lm, N, dtype=torch.complex128) for _ in range(6)]
    ub.updateB(*bj, tb, tj, tscheme)
    for f, ta_, (x, dx, d2x) in (("b", tb, bj[:3]), ("j", tj, bj[3:])):
        out.update({f + "_new": n(x), "d" + f + "_new": n(dx), "dd" + f + "_new": n(d2x),
                    f + "_impl_new": n(ta_.impl[:, :, 0]), f + "_old_new": n(ta_.old[:, :, 0]),
                    f + "_expl1_new": n(ta_.expl[:, :, 1])})
    if params.l_double_curl:
        # one double-curl poloidal update with the l = 0 pressure
        # (magic_torch/update_w_doublecurl.py:67-483, update_wp.py:80-194)
        from magic_torch import update_w_doublecurl as uw, update_wp as uwp
        uw.build_w_matrices(tscheme.wimp_lin[0].item())
        uwp.build_p0_matrix()
        tw = dtf.TimeArray(tscheme.nold, tscheme.nexp, tscheme.nimp)
        for k in ("old", "impl", "expl0", "expl1"):
            v = _spec(rng, lm, l_of, N)
            (tw.old if k == "old" else tw.impl if k == "impl" else tw.expl)[
                :, :, 1 if k == "expl1" else 0] = t(v)
            out["w_" + k] = v
        out.update(rgrav=n(rf2.rgrav), rho0=n(rf2.rho0), ddbeta=n(rf2.ddbeta),
                   ddLvisc=n(rf2.ddLvisc), BuoFac=float(pc.BuoFac), ChemFac=float(pc.ChemFac),
                   d3rMat=n(rs.d3rMat), d4rMat=n(rs.d4rMat))
        w_new, dw_new, ddw_new, p_new, dp_new = (torch.zeros(lm, N, dtype=torch.complex128)
                                                 for _ in range(5))
        uw.updateW(s_new.clone(), w_new, dw_new, ddw_new, tw, p_new, dp_new, tscheme)
        out.update(w_new=n(w_new), dw_new=n(dw_new), ddw_new=n(ddw_new), p0_new=n(p_new[0]),
                   w_impl_new=n(tw.impl[:, :, 0]), w_old_new=n(tw.old[:, :, 0]),
                   w_expl1_new=n(tw.expl[:, :, 1]))
    else:
        # one coupled (w, p) update in the standard form with the l = 0 pressure
        # (magic_torch/update_wp.py:80-531)
        from magic_torch import update_wp as uwp
        uwp.build_wp_matrices(tscheme.wimp_lin[0].item())
        uwp.build_p0_matrix()
        tw = dtf.TimeArray(tscheme.nold, tscheme.nexp, tscheme.nimp)
        tp = dtf.TimeArray(tscheme.nold, tscheme.nexp, tscheme.nimp)
        for f, ta_ in (("wp_w", tw), ("wp_p", tp)):
            for k in ("old", "impl", "expl0", "expl1"):
                v = _spec(rng, lm, l_of, N)
                (ta_.old if k == "old" else ta_.impl if k == "impl" else ta_.expl)[
                    :, :, 1 if k == "expl1" else 0] = t(v)
                out[f + "_" + k] = v
        out.update(rgrav=n(rf2.rgrav), rho0=n(rf2.rho0), BuoFac=float(pc.BuoFac),
                   d3rMat=n(rs.d3rMat), D3=n(rd._D3_real))
        w_new, dw_new, ddw_new, p_new, dp_new = (torch.zeros(lm, N, dtype=torch.complex128)
                                                 for _ in range(5))
        uwp.updateWP(s_new.clone(), w_new, dw_new, ddw_new, tw, p_new, dp_new, tp, tscheme)
        out.update({"wp_w_new": n(w_new), "wp_dw_new": n(dw_new), "wp_ddw_new": n(ddw_new),
                    "wp_p_new": n(p_new), "wp_dp_new": n(dp_new)})
        for f, ta_ in (("wp_w", tw), ("wp_p", tp)):
            out.update({f + "_impl_new": n(ta_.impl[:, :, 0]), f + "_old_new": n(ta_.old[:, :, 0]),
                        f + "_expl1_new": n(ta_.expl[:, :, 1])})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def worker_energy(name, ref):
    cfg = dict(ENERGY_CONFIGS[name], device="cpu", use_shtns=False)
    sys.path.insert(0, ref)
    from magic_torch.config import configure
    configure(cfg)
    import torch
    from magic_torch import params, blocking, radial_functions as rf, pre_calculations as pc
    from magic_torch.radial_scheme import r as r_grid
    from magic_torch.output import get_e_kin_full, get_e_mag_oc_full
    from magic_torch.integration import rInt_R
    n = lambda x: x.detach().cpu().numpy().copy()
    rng = np.random.default_rng(99)
    N, lm = params.n_r_max, params.lm_max
    l_of = n(blocking.st_lm2l)
    m_of = n(blocking.st_lm2m)
    ins = {k: _spec(rng, lm, l_of, N) for k in ("w", "dw", "z", "b", "db", "aj")}
    for k in ins:
        ins[k][m_of == 0] = ins[k][m_of == 0].real
    T = {k: torch.from_numpy(v) for k, v in ins.items()}
    out = dict(n_r_max=N, l_max=params.l_max, minc=params.minc, lm_max=lm, lm2l=l_of, lm2m=m_of,
               r=n(r_grid), or2=n(rf.or2), orho1=n(rf.orho1), LFfac=float(pc.LFfac),
               radratio=float(params.radratio), chebyshev=int(params.radial_scheme != "FD"),
               rint_w=n(rInt_R(torch.eye(N, dtype=torch.float64))),
               e_kin=np.array(get_e_kin_full(T["w"], T["dw"], T["z"])),
               e_mag=np.array(get_e_mag_oc_full(T["b"], T["db"], T["aj"])))
    out.update({"in_" + k: v for k, v in ins.items()})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def worker_step(name, ref):
    """Reference state before and after two one_step calls, the reference's own
    checkpoint dictionary layout (main.py:189-222), kinetic and magnetic
    energies (output.py:101-180) and the radial integration weights."""
    import json
    import tempfile

    cfg = dict(STEP_CONFIGS[name], device="cpu", use_shtns=False)
    sys.path.insert(0, ref)
    from magic_torch.config import configure
    configure(cfg)
    import torch
    from magic_torch import params, blocking, fields
    from magic_torch.init_fields import initialize_fields
    from magic_torch.step_time import setup_initial_state, one_step, initialize_dt
    from magic_torch.main import save_checkpoint
    from magic_torch.output import get_e_kin_full, get_e_mag_oc_full
    from magic_torch.integration import rInt_R
    from magic_torch.time_scheme import tscheme
    n = lambda x: x.detach().cpu().numpy().copy()
    N, lm = params.n_r_max, params.lm_max
    initialize_fields()
    # seeded perturbations on the interior levels (m = 0 real), so that every
    # nonlinear and Coriolis term is active in the first step
    g = torch.Generator().manual_seed(11)
    m0 = blocking.st_lm2m == 0
    for fld, amp in (("s_LMloc", 1e-3), ("w_LMloc", 1e-3), ("z_LMloc", 1e-3)):
        c = torch.complex(torch.randn(lm, N, generator=g, dtype=torch.float64),
                          torch.randn(lm, N, generator=g, dtype=torch.float64)) * amp
        c[m0] = c[m0].real.to(c.dtype)
        getattr(fields, fld)[:, 1:-1] += c[:, 1:-1]
    setup_initial_state()
    dt = float(cfg["dtmax"])
    initialize_dt(dt)
    out = dict(n_r_max=N, l_max=params.l_max, minc=params.minc, lm_max=lm, dt=dt,
               ek=cfg["ek"], ra=cfg["ra"], pr=cfg["pr"], prmag=cfg["prmag"],
               radratio=float(params.radratio), lm2l=n(blocking.st_lm2l),
               lm2m=n(blocking.st_lm2m))
    rint = rInt_R(torch.eye(N, dtype=torch.float64))
    out["rint_w"] = n(rint)
    if params.l_anel:
        # the anelastic background and the angular-momentum constants the step uses
        from magic_torch import radial_functions as rf, pre_calculations as pc
        from magic_torch.radial_scheme import r as r_grid
        out.update(r=n(r_grid), rho0=n(rf.rho0), beta=n(rf.beta), dbeta=n(rf.dbeta),
                   rgrav=n(rf.rgrav), dLtemp0=n(rf.dLtemp0), otemp1=n(rf.otemp1),
                   ViscHeatFac=float(rf.ViscHeatFac), c_moi_oc=float(pc.c_moi_oc),
                   cfg=json.dumps(cfg))

    def snapshot(tag, fields_only=None):
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "ck.pt")
            save_checkpoint(path, 0, 0.0, {"tag": "golden"})
            st = torch.load(path, weights_only=False)
        if tag == "0":
            out["ckpt_layout"] = json.dumps({k: (list(v.shape) if torch.is_tensor(v)
                                                 else type(v).__name__)
                                             for k, v in st.items()})
        for k, v in st.items():
            if not torch.is_tensor(v) or v.dim() < 2:
                continue
            if fields_only and k not in fields_only:
                continue
            out[tag + ":" + k] = n(v)
        w, dw, z = fields.w_LMloc, fields.dw_LMloc, fields.z_LMloc
        out[tag + ":e_kin"] = np.array(get_e_kin_full(w, dw, z))
        out[tag + ":e_mag"] = np.array(get_e_mag_oc_full(fields.b_LMloc, fields.db_LMloc,
                                                         fields.aj_LMloc))
        out[tag + ":tscheme_dt"] = n(tscheme.dt)

    snapshot("0")
    for step in (1, 2):
        dt_new = one_step(step, dt)
        assert dt_new == dt, (dt_new, dt)
        snapshot(str(step), fields_only=None if step == 2 else (
            "fields.w_LMloc", "fields.z_LMloc", "fields.s_LMloc", "fields.b_LMloc",
            "fields.aj_LMloc"))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def worker_run(name, ref):
    """The reference's own initial state (initialize_fields + seeded entropy
    noise + setup_initial_state, saved through save_checkpoint), its kinetic and
    magnetic energies after every one_step call, and its fields after the last
    step, all at a fixed dt (the run asserts that the Courant check never changed
    it)."""
    import tempfile

    cfg, nsteps, noise = RUN_CONFIGS[name]
    cfg = dict(cfg, device="cpu", use_shtns=False)
    sys.path.insert(0, ref)
    from magic_torch.config import configure
    configure(cfg)
    import torch
    from magic_torch import params, blocking, fields
    from magic_torch.init_fields import initialize_fields
    from magic_torch.step_time import setup_initial_state, one_step, initialize_dt
    from magic_torch.main import save_checkpoint
    from magic_torch.output import get_e_kin_full, get_e_mag_oc_full
    from magic_torch.time_scheme import tscheme
    n = lambda x: x.detach().cpu().numpy().copy()
    N, lm = params.n_r_max, params.lm_max
    initialize_fields()
    g = torch.Generator().manual_seed(0)
    m0 = blocking.st_lm2m == 0
    c = torch.complex(torch.randn(lm, N, generator=g, dtype=torch.float64),
                      torch.randn(lm, N, generator=g, dtype=torch.float64)) * noise
    c[m0] = c[m0].real.to(c.dtype)
    fields.s_LMloc[:, 1:-1] += c[:, 1:-1]
    setup_initial_state()
    dt = float(cfg["dtmax"])
    initialize_dt(dt)
    out = dict(n_r_max=N, l_max=params.l_max, minc=params.minc, lm_max=lm, dt=dt,
               ek=cfg["ek"], ra=cfg["ra"], pr=cfg["pr"], prmag=cfg["prmag"],
               radratio=float(params.radratio), steps=nsteps, noise=noise)
    if params.l_anel:
        import json
        out["cfg"] = json.dumps(cfg)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "ck.pt")
        save_checkpoint(path, 0, 0.0, {"tag": "golden"})
        st = torch.load(path, weights_only=False)
    for k, v in st.items():
        if torch.is_tensor(v) and v.dim() >= 2:
            out["0:" + k] = n(v)
    out["0:tscheme_dt"] = n(tscheme.dt)
    ek_t, em_t = [], []
    for step in range(1, nsteps + 1):
        dt_new = one_step(step, dt)
        assert dt_new == dt, (step, dt_new, dt)
        ek_t.append(np.array(get_e_kin_full(fields.w_LMloc, fields.dw_LMloc, fields.z_LMloc)))
        em_t.append(np.array(get_e_mag_oc_full(fields.b_LMloc, fields.db_LMloc,
                                               fields.aj_LMloc)))
    out["e_kin"], out["e_mag"] = np.stack(ek_t), np.stack(em_t)
    for k in ("w", "z", "s", "p", "b", "aj"):
        out[f"{nsteps}:{k}"] = n(getattr(fields, k + "_LMloc"))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def worker_adapt(name, ref):
    """The reference's initial state (initialize_fields, seeded perturbations of
    s, w and z as worker_step draws them, setup_initial_state), then one_step with
    the Courant control: the dt of every step, the energies after every step and
    the fields after the last."""
    import tempfile

    cfg, nsteps = ADAPT_CONFIGS[name]
    cfg = dict(cfg, device="cpu", use_shtns=False)
    sys.path.insert(0, ref)
    from magic_torch.config import configure
    configure(cfg)
    import torch
    from magic_torch import params, blocking, fields
    from magic_torch.init_fields import initialize_fields
    from magic_torch.step_time import setup_initial_state, one_step, initialize_dt
    from magic_torch.main import save_checkpoint
    from magic_torch.output import get_e_kin_full, get_e_mag_oc_full
    from magic_torch.time_scheme import tscheme
    n = lambda x: x.detach().cpu().numpy().copy()
    N, lm = params.n_r_max, params.lm_max
    initialize_fields()
    g = torch.Generator().manual_seed(11)
    m0 = blocking.st_lm2m == 0
    for fld, amp in (("s_LMloc", 1e-3), ("w_LMloc", 1e-3), ("z_LMloc", 1e-3)):
        c = torch.complex(torch.randn(lm, N, generator=g, dtype=torch.float64),
                          torch.randn(lm, N, generator=g, dtype=torch.float64)) * amp
        c[m0] = c[m0].real.to(c.dtype)
        getattr(fields, fld)[:, 1:-1] += c[:, 1:-1]
    setup_initial_state()
    dt = float(cfg["dtmax"])
    initialize_dt(dt)
    out = dict(n_r_max=N, l_max=params.l_max, minc=params.minc, lm_max=lm, dtmax=dt,
               ek=cfg["ek"], ra=cfg["ra"], pr=cfg["pr"], prmag=cfg["prmag"],
               radratio=float(params.radratio), steps=nsteps)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "ck.pt")
        save_checkpoint(path, 0, 0.0, {"tag": "golden"})
        st = torch.load(path, weights_only=False)
    for k, v in st.items():
        if torch.is_tensor(v) and v.dim() >= 2:
            out["0:" + k] = n(v)
    out["0:tscheme_dt"] = n(tscheme.dt)
    dts, ek_t, em_t = [], [], []
    for step in range(1, nsteps + 1):
        dt = one_step(step, dt)
        dts.append(dt)
        ek_t.append(np.array(get_e_kin_full(fields.w_LMloc, fields.dw_LMloc, fields.z_LMloc)))
        em_t.append(np.array(get_e_mag_oc_full(fields.b_LMloc, fields.db_LMloc,
                                               fields.aj_LMloc)))
    out["dt"], out["e_kin"], out["e_mag"] = np.array(dts), np.stack(ek_t), np.stack(em_t)
    for k in ("w", "z", "s", "p", "b", "aj"):
        out[f"{nsteps}:{k}"] = n(getattr(fields, k + "_LMloc"))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference/src")
    ap.add_argument("--worker", default=None)
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    if a.worker:
        if a.worker in SHT_CONFIGS:
            worker_sht(a.worker, a.ref)
        elif a.worker in TD_CONFIGS:
            worker_td(a.worker, a.ref)
        elif a.worker in STEP_CONFIGS:
            worker_step(a.worker, a.ref)
        elif a.worker in RUN_CONFIGS:
            worker_run(a.worker, a.ref)
        elif a.worker in ADAPT_CONFIGS:
            worker_adapt(a.worker, a.ref)
        elif a.worker in ENERGY_CONFIGS:
            worker_energy(a.worker, a.ref)
        else:
            worker_nl(a.worker, a.ref)
        return
    env = dict(os.environ, TORCHDYNAMO_DISABLE="1", MAGIC_DEVICE="cpu")
    names = list(SHT_CONFIGS) + list(NL_CONFIGS) + list(TD_CONFIGS) + list(STEP_CONFIGS)
    names += list(ENERGY_CONFIGS) + list(RUN_CONFIGS) + list(ADAPT_CONFIGS)
    if a.only:
        names = [x for x in names if x in a.only.split(",")]
    for name in names:
        print("golden:", name, flush=True)
        subprocess.run([sys.executable, os.path.abspath(__file__), "--worker", name,
                        "--ref", a.ref], check=True, env=env, cwd="/tmp")


if __name__ == "__main__":
    main()
