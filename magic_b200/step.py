"""One CNAB2 time step of the Boussinesq dynamo on the GPU.

The reference's one_step (magic_torch/step_time.py:1574-1640) with its
radial_loop (:931-1213) and lm_loop (:1478-1527), for the finite-difference
radial scheme with the double-curl poloidal form or the Chebyshev scheme with
the standard coupled (w, p) form (the reference ties the form to the scheme,
params.py:143), an insulating inner core and mantle, Boussinesq profiles,
magnetic field on:

    radial loop  mt_nl_bouss (input assembly, synthesis, phi FFT, get_nl
                 products, Courant, analysis) then mt_get_td (explicit terms
                 with finish_exp), written straight into each field's expl0;
    lm loop      entropy (mt_update_field), toroidal velocity
                 (mt_update_field), poloidal velocity and l = 0 pressure
                 (mt_update_poloidal, double curl; mt_update_wp, standard
                 form with the pressure of every degree), magnetic b and j
                 (mt_update_field), in the reference's order S, Z, W, B.

By default the time step is held fixed (the solve operators are built once
for it) and the Courant limits of every step are returned; step(adaptive=True)
applies the reference's Courant control of dt instead.
Every launch is stream-ordered on the current stream; nothing synchronises.
"""

import math

import numpy as np
import torch

from . import implicit as I
from .plan import Plan
from .radial import RadialOp, RadialScheme

_CD = torch.complex128


def dt_courant(dt, dt_max, dt_min):
    """(changed, dt_new) of the reference's Courant control of dt
    (magic_torch/courant.py:130-155) for the current step dt and the smallest
    Courant limit dt_min over the levels: with dt_2 = min(0.75 dt_min, dt_max), a
    step above dt_max falls to dt_max, a step above the limit to dt_2, and a step
    below half the limit (and below dt_max) rises to dt_2."""
    dt_2 = min(0.5 * (1.0 / 2.0 + 1.0) * dt_min, dt_max)
    if dt > dt_max:
        return True, dt_max
    if dt > dt_min:
        return True, dt_2
    if 2.0 * dt < dt_min and dt < dt_max:
        return True, dt_2
    return False, dt


class BoussinesqStep:
    l_mag = True        # magnetic field on (subclasses may turn it off)
    l_anel = False      # anelastic background and terms
    am = None           # angular-momentum corrections of z (AnelasticStep)

    def __init__(self, l_max, n_r, ek=1e-5, ra=3e8, pr=1.0, prmag=1.0, dt=2e-7,
                 precision="split", radratio=0.35, fd_order=4, fd_order_bound=2, ktopv=2,
                 kbotv=2, device=None, cache=None, minc=1, radial_scheme="FD"):
        """minc: azimuthal symmetry (orders m = 0, minc, 2 minc, ...; the grid covers
        one sector of 2 pi / minc).  radial_scheme: "FD" (fourth-order by default,
        double-curl poloidal form) or "chebyshev" (n_r Gauss-Lobatto levels,
        standard (w, p) form).

        cache: optional dict shared by several steps on one device; the read-only
        parts that depend only on the grid and the dt pair (transform plan, radial
        operators, per-degree solve operators) are taken from it or added to it, so
        runs of the same shape share one resident copy."""
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        dev = self.device
        self._cache = cache if cache is not None else {}
        self.std_form = radial_scheme.upper() != "FD"
        self._shape = (n_r, radial_scheme.upper(), radratio, fd_order, fd_order_bound, str(dev)) \
            + self._background_key()
        self.plan = self._shared(("plan", l_max, minc, precision, str(dev)),
                                 lambda: Plan(l_max, minc, precision=precision, device=dev))
        self.sch = self._shared(("sch",) + self._shape,
                                lambda: RadialScheme(n_r, radial_scheme, radratio,
                                                     fd_order=fd_order,
                                                     fd_order_bound=fd_order_bound, device=dev))
        self.l_max, self.n_r, self.lm_max = l_max, n_r, self.plan.lm_max
        # physical prefactors (magic_torch/pre_calculations.py:13-41)
        self.CorFac, self.LFfac = 1.0 / ek, 1.0 / (ek * prmag)
        self.BuoFac, self.opr, self.opm = ra / pr, 1.0 / pr, 1.0 / prmag
        r = self.sch.r
        r_cmb = 1.0 / (1.0 - radratio)
        dr = np.abs(np.diff(r))
        delxr2 = np.empty(n_r)
        delxr2[0], delxr2[-1] = dr[0] ** 2, dr[-1] ** 2
        delxr2[1:-1] = np.minimum(dr[:-1], dr[1:]) ** 2
        zeros, ones = np.zeros(n_r), np.ones(n_r)
        hp = dict(r=r, or1=1.0 / r, or2=1.0 / r ** 2, or4=1.0 / r ** 4, orho1=ones,
                  orho2=ones, beta=zeros, dbeta=zeros, ddbeta=zeros, visc=ones, dLvisc=zeros,
                  ddLvisc=zeros, kappa=ones, dLkappa=zeros, dLtemp0=zeros, lambda_=ones,
                  dLlambda=zeros, rgrav=r / r_cmb, rho0=ones, otemp1=ones, delxr2=delxr2,
                  delxh2=r ** 2 / float(l_max * (l_max + 1)))
        hp.update(self._background(r, radratio, ek=ek, ra=ra, pr=pr, prmag=prmag))
        self.hprof = hp
        t = lambda x: torch.as_tensor(np.asarray(x, dtype=np.float64), device=dev).contiguous()
        self.prof = {k: t(v) for k, v in hp.items()}
        hdif = np.ones(l_max + 1)
        self.hdif = t(hdif)
        self._hdif_np, self._ktopv, self._kbotv = hdif, ktopv, kbotv
        d1c = hp["beta"] + hp["dLtemp0"] + 2.0 * hp["or1"] + hp["dLkappa"]
        self._d1c = d1c
        # CNAB2 weights and the per-degree solve operators of the current dt pair
        self.dt = None
        self.dt_max = float(dt)  # the Courant control's upper bound (initialize_dt)
        self.set_dt(dt, dt)
        pc = self._p0_constraint()
        self.P0 = self._shared(("P0",) + self._shape,
                               lambda: RadialOp(I.p0_inverse(self.sch, hp["beta"],
                                                             pc[0] if pc else None), device=dev))
        self.p0_row0 = t(pc[1]) if pc else None
        dev_coef = lambda c: {k: (t(v) if v is not None else None) for k, v in c.items()}
        self.coef = dict(s=dev_coef(I.entropy_coefficients(l_max, self.opr, hdif, hp["kappa"],
                                                           self._d1c, hp["or2"])),
                         z=dev_coef(I.toroidal_coefficients(l_max, hdif, hp["visc"], hp["beta"],
                                                            hp["dbeta"], hp["dLvisc"], hp["or1"],
                                                            hp["or2"])))
        if self.l_mag:
            cb, cj = I.magnetic_coefficients(l_max, self.opm, hdif, hp["lambda_"],
                                             hp["dLlambda"], hp["or2"])
            self.coef["b"], self.coef["j"] = dev_coef(cb), dev_coef(cj)
        self.wprof = {k: self.prof[k] for k in ("or1", "or2", "beta", "dbeta", "ddbeta", "visc",
                                                "dLvisc", "ddLvisc", "orho1", "rgrav", "rho0")}
        self.wcoef = tuple(t(c) for c in I._w_coefficient_profiles(hp))
        self.wpprof = {k: self.prof[k] for k in ("or1", "or2", "beta", "dbeta", "visc", "dLvisc",
                                                 "rgrav", "rho0")}
        # state: fields, their derivatives and the time arrays of each equation
        z = lambda: torch.zeros(self.lm_max, n_r, dtype=_CD, device=dev)
        mag = self.l_mag
        self.f = {k: z() for k in ("w", "dw", "ddw", "z", "dz", "s", "ds", "p")
                  + (("b", "db", "ddb", "aj", "dj", "ddj") if mag else ())
                  + (("dp",) if self.std_form else ())}
        self.ta = {e: {k: z() for k in ("old", "impl", "expl0", "expl1")}
                   for e in ("s", "z", "w") + (("b", "j") if mag else ())
                   + (("p",) if self.std_form else ())}
        self.nl_out = {k: z() for k in self.stage_outputs()}
        self._work = None  # the stage workspace, allocated at the first own stage
        self.bots = torch.zeros(self.lm_max, dtype=_CD, device=dev)
        self.bots[0] = math.sqrt(4.0 * math.pi)  # fixed entropy at the inner boundary, l = m = 0

    def set_dt(self, dt_new, dt_old):
        """CNAB2 weights for the step dt_new after dt_old (time_scheme.py:56-73) and,
        when the implicit weight changed, new solve operators (the reference's
        build_all_matrices, step_time.py:1625-1627)."""
        if self.dt == (float(dt_new), float(dt_old)):
            return
        self.dt = (float(dt_new), float(dt_old))
        self.weights = I.cnab2_weights(*self.dt)
        wl0 = self.weights[1]
        if getattr(self, "_ops_wl0", None) == wl0:
            return
        key = ("ops", self.l_max, wl0, self.opr, self.opm, self._ktopv, self._kbotv) + self._shape
        self.ops = self._shared(key, lambda: self._build_ops(wl0))
        self._ops_wl0 = wl0

    def _background_key(self):
        """Parameters of the radial background beyond the grid (cache key part)."""
        return ()

    def _background(self, r, radratio, **phys):
        """Radial profiles replacing the Boussinesq ones (none here)."""
        return {}

    def _p0_constraint(self):
        """(matrix row weights, right-hand-side weights) of an integral constraint
        replacing p = 0 in the l = 0 pressure equation, or None."""
        return None

    def stage_outputs(self):
        """Spectral outputs of this step's nonlinear stage."""
        return self.STAGE_OUTPUTS

    def _shared(self, key, build):
        if key not in self._cache:
            self._cache[key] = build()
        return self._cache[key]

    def _build_ops(self, wl0):
        hp, hdif, dev, l_max = self.hprof, self._hdif_np, self.device, self.l_max
        ops = dict(
            s=I.LOp(I.scalar_solve_operators(self.sch, l_max, wl0, self.opr, hdif, hp["kappa"],
                                             self._d1c, hp["or2"]), device=dev),
            z=I.LOp(I.toroidal_solve_operators(self.sch, l_max, wl0, hdif, hp["visc"],
                                               hp["beta"], hp["dbeta"], hp["dLvisc"], hp["or1"],
                                               hp["or2"], self._ktopv, self._kbotv), device=dev),
            w=I.LOp(I.wp_solve_operators(self.sch, l_max, wl0, hdif, hp, self._ktopv,
                                         self._kbotv) if self.std_form else
                    I.poloidal_dc_solve_operators(self.sch, l_max, wl0, hdif, hp, self._ktopv,
                                                  self._kbotv), device=dev))
        if self.l_mag:
            Mb, Mj = I.magnetic_solve_operators(self.sch, l_max, wl0, self.opm, hdif,
                                                hp["lambda_"], hp["dLlambda"], hp["or1"],
                                                hp["or2"])
            ops["b"], ops["j"] = I.LOp(Mb, device=dev), I.LOp(Mj, device=dev)
        return ops

    def energies(self):
        """Kinetic and magnetic energies of the current state (EKin, EMagOC of
        magic_torch/output.py:101-190), computed on the GPU in FP64."""
        from .output import EnergyIntegrals

        if not hasattr(self, "_energy"):
            hp = self.hprof
            self._energy = EnergyIntegrals(self.plan, hp["r"], hp["or2"], hp["orho1"],
                                           self.sch.rint, self.LFfac)
        f = self.f
        kin = self._energy.kin(f["w"], f["dw"], f["z"])
        if not self.l_mag:
            return kin, np.zeros(12)
        return kin, self._energy.mag(f["b"], f["db"], f["aj"])

    def init_random(self, seed=0, amp=1e-4):
        """Seeded random fields |c_lm| ~ amp (l+1)^-2 on the interior levels (m = 0
        real), their radial derivatives, and the old / implicit time arrays built from
        them as the reference's setup_initial_state does (step_time.py:398-600: old =
        s, l(l+1)/r^2 z, the double-curl w term, l(l+1)/r^2 b and j; impl = each
        equation's implicit operator applied to the fields)."""
        from .radial import get_ddr

        # drawn on the device (a CPU draw of these arrays dominated the build of a
        # run); the same seed gives the same fields on a given device type
        dev = self.device
        g = torch.Generator(device=dev).manual_seed(seed)
        decay = (torch.as_tensor(self.plan.lm2l, dtype=torch.float64, device=dev) + 1.0) ** -2
        m0 = torch.as_tensor(self.plan.lm2m == 0, device=dev)
        for k in ("w", "z", "s", "b", "aj"):
            c = torch.randn(self.lm_max, self.n_r, dtype=_CD, generator=g, device=dev) * amp
            if k not in self.f:
                continue
            c *= decay[:, None]
            c[m0] = c[m0].real.to(_CD)
            c[:, 0] = 0.0
            c[:, -1] = 0.0
            self.f[k].copy_(c)
        f, P, D1, D2 = self.f, self.prof, self.sch.D1, self.sch.D2
        second = {}
        for k, d1, d2 in (("w", "dw", "ddw"), ("z", "dz", None), ("s", "ds", None),
                          ("b", "db", "ddb"), ("aj", "dj", "ddj")):
            if k not in f:
                continue
            a1, a2 = get_ddr(f[k], D1, D2)
            f[d1].copy_(a1)
            second[k] = a2
            if d2:
                f[d2].copy_(a2)
        l = torch.as_tensor(self.plan.lm2l, dtype=torch.float64, device=self.device)
        dL = (l * (l + 1.0))[:, None]
        row = lambda x: x[None, :]
        hd = self.hdif[self.plan_l()][:, None]

        def generic(key, x, dx, d2x):
            c = self.coef[key]
            so = (c["so_l"][self.plan_l()][:, None] * row(c["so_r"])) if c["so_l"] is not None \
                else 1.0
            ic = (row(c["ic_r"]) if c["ic_r"] is not None else 0.0) \
                + c["ic_l"][self.plan_l()][:, None] * row(c["ic_r2"])
            impl = c["ia_l"][self.plan_l()][:, None] * row(c["ia_r"]) * (
                d2x + row(c["ib_r"]) * dx - ic * x)
            self.ta[key]["old"].copy_(so * x)
            self.ta[key]["impl"].copy_(impl)

        generic("s", f["s"], f["ds"], second["s"])
        generic("z", f["z"], f["dz"], second["z"])
        if self.l_mag:
            generic("b", f["b"], f["db"], second["b"])
            generic("j", f["aj"], f["dj"], second["aj"])
        if self.std_form:
            self._init_wp_terms(dL, hd)
            return
        # double-curl poloidal terms (update_w_doublecurl.py:310-390)
        dddw, ddddw = get_ddr(f["ddw"], D1, D2)
        or2, orho1, beta = row(P["or2"]), row(P["orho1"]), row(P["beta"])
        old = dL * or2 * (-orho1 * (f["ddw"] - beta * f["dw"] - dL * or2 * f["w"]))
        c3, c2n, c1n, c1d, c0n = (row(c) for c in self.wcoef)
        dLo = dL * or2
        dif = -hd * dLo * row(P["visc"]) * orho1 * (
            ddddw + c3 * dddw + (c2n - 2.0 * dLo) * f["ddw"] + (c1n + dL * c1d) * f["dw"]
            + dLo * (c0n + dLo) * f["w"])
        impl = dif + self.BuoFac * dLo * row(P["rgrav"]) * f["s"]
        for x in (old, impl):
            x[:, 0] = 0.0
            x[:, -1] = 0.0
        self.ta["w"]["old"].copy_(old)
        self.ta["w"]["impl"].copy_(impl)

    def _init_wp_terms(self, dL, hd):
        """old and implicit terms of the standard-form w and p equations from the
        current fields (step_time.py:491-545): dwdt.old = l(l+1) or2 w, dpdt.old =
        -l(l+1) or2 dw, and the implicit operators of update_wp.py:492-531 (row 0
        of the lm order is (l, m) = (0, 0))."""
        f, P = self.f, self.prof
        row = lambda x: x[None, :]
        dddw = self.sch.D3(f["w"])
        f["dp"].copy_(self.sch.D1(f["p"]))
        or1, or2, beta, dbeta = (row(P[k]) for k in ("or1", "or2", "beta", "dbeta"))
        visc, dLv = row(P["visc"]), row(P["dLvisc"])
        dLo = dL * or2
        w, dw, ddw, p, dp = f["w"], f["dw"], f["ddw"], f["p"], f["dp"]
        dif = hd * dLo * visc * (ddw + (2.0 * dLv - beta / 3.0) * dw - (
            dLo + 4.0 / 3.0 * (dbeta + dLv * beta + (3.0 * dLv + beta) * or1)) * w)
        self.ta["w"]["old"].copy_(dLo * w)
        self.ta["w"]["impl"].copy_(-dp + beta * p + dif
                                   + self.BuoFac * row(P["rho0"]) * row(P["rgrav"]) * f["s"])
        self.ta["p"]["old"].copy_(-dLo * dw)
        self.ta["p"]["impl"].copy_(dLo * p + hd * visc * dLo * (
            -dddw + (beta - dLv) * ddw + (dLo + dLv * beta + dbeta + 2.0 * (dLv + beta) * or1) * dw
            - dLo * (2.0 * or1 + 2.0 / 3.0 * beta + dLv) * w))
        # l = 0 and the boundary levels zero (step_time.py:538-545)
        for e in ("w", "p"):
            x = self.ta[e]["impl"]
            x[0] = 0.0
            x[:, 0] = 0.0
            x[:, -1] = 0.0

    def plan_l(self):
        if not hasattr(self, "_l_dev"):
            self._l_dev = torch.as_tensor(self.plan.lm2l, dtype=torch.long, device=self.device)
        return self._l_dev

    @property
    def work(self):
        """Workspace of this step's own fused stage (runs whose stage is shared
        with other runs never allocate it)."""
        if self._work is None:
            self._work = torch.empty(self.plan.nl_bouss_workspace(self.n_r, True, False),
                                     dtype=torch.uint8, device=self.device)
        return self._work

    STAGE_INPUTS = ("w", "dw", "ddw", "z", "dz", "s", "b", "db", "ddb", "aj", "dj")
    STAGE_OUTPUTS = ("Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt", "VxBp")

    def radial_loop(self):
        """Explicit stage: nonlinear products and Courant limits, then the explicit
        time derivatives into each equation's expl0 (step_time.py:931-1213)."""
        dtr, dth = self.nonlinear_stage()
        self.explicit_terms()
        return dtr, dth

    def nonlinear_stage(self):
        """The fused nonlinear stage of the radial loop into self.nl_out; returns
        the per-level Courant steps (dtrkc, dthkc)."""
        f = self.f
        fields = {k: f[k] for k in self.STAGE_INPUTS}
        _, dtr, dth = self.plan.nl_bouss(fields, self.prof, self.LFfac, 2.5, 1.0, self.opm,
                                         l_mag=True, out=self.nl_out, work=self.work)
        return dtr, dth

    def explicit_terms(self):
        """get_td + finish_exp from self.nl_out (whoever filled it: this step's own
        stage, or a stage shared by several runs) into each equation's expl0."""
        f = self.f
        ins = dict(self.nl_out, w=f["w"], dw=f["dw"], ddw=f["ddw"], z=f["z"], dz=f["dz"])
        td_out = dict(dwdt=self.ta["w"]["expl0"], dzdt=self.ta["z"]["expl0"],
                      dsdt=self.ta["s"]["expl0"])
        if self.l_mag:
            td_out.update(dbdt=self.ta["b"]["expl0"], djdt=self.ta["j"]["expl0"])
        if self.std_form:
            td_out["dpdt"] = self.ta["p"]["expl0"]
        self.plan.get_td(ins, self.prof, self.CorFac, self.sch.D1,
                         l_double_curl=not self.std_form, l_heat=True, l_mag=self.l_mag,
                         l_anel=self.l_anel, out=td_out)

    def lm_loop(self):
        """Implicit solves S, Z, W, B (step_time.py:1478-1527).  The Boussinesq
        standard form stores its implicit terms zero at l = 0 and on the boundary
        levels, as the reference's fused lm loop does (:380-394); the anelastic
        loop calls updateWP itself, which stores every entry (update_wp.py:
        491-531; neither affects the solution)."""
        f, ta, w = self.f, self.ta, self.weights
        I.update_field(self.plan, self.sch, self.ops["s"], f["s"], f["ds"], ta["s"], w,
                       self.coef["s"], bot=self.bots)
        I.update_field(self.plan, self.sch, self.ops["z"], f["z"], f["dz"], ta["z"], w,
                       self.coef["z"])
        if self.am is not None:
            I.correct_am(self.plan, f["z"], f["dz"], ta["z"], self.coef["z"], self.am)
        if self.std_form:
            I.update_wp(self.plan, self.sch, self.ops["w"], self.P0, f["w"], f["dw"], f["ddw"],
                        f["p"], f["dp"], ta["w"], ta["p"], w, f["s"], self.wpprof, self.hdif,
                        self.BuoFac, impl_interior=not self.l_anel, p0_row0=self.p0_row0)
        else:
            I.update_poloidal_dc(self.plan, self.sch, self.ops["w"], self.P0, f["w"], f["dw"],
                                 f["ddw"], f["p"], ta["w"], w, f["s"], self.wprof, self.hdif,
                                 self.BuoFac, wcoef=self.wcoef)
        if not self.l_mag:
            return
        I.update_field(self.plan, self.sch, self.ops["b"], f["b"], f["db"], ta["b"], w,
                       self.coef["b"], d2x=f["ddb"])
        I.update_field(self.plan, self.sch, self.ops["j"], f["aj"], f["dj"], ta["j"], w,
                       self.coef["j"], d2x=f["ddj"])

    def courant_dt(self, dtr, dth):
        """(changed, dt_new) of the Courant control (dt_courant) from the per-level
        limits of this step's radial loop.  Reads the minima on the host (one
        synchronisation, as the reference's .item())."""
        return dt_courant(self.dt[0], self.dt_max, min(float(dtr.min()), float(dth.min())))

    def step(self, adaptive=False):
        """One CNAB2 step.  adaptive: the reference's one_step order
        (step_time.py:1602-1633): radial loop, Courant decision, dt history rolled
        and the CNAB2 weights (and, when the step size changed, the solve
        operators) renewed, then the lm loop; the default keeps dt fixed and never
        synchronises."""
        dtr, dth = self.radial_loop()
        if adaptive:
            _, dt_new = self.courant_dt(dtr, dth)
            self.set_dt(dt_new, self.dt[0])
        self.lm_loop()
        return dtr, dth


class AnelasticStep(BoussinesqStep):
    """One CNAB2 step of anelastic convection on the GPU: the reference's one_step
    (magic_torch/step_time.py:1574-1640) with radial_loop_anel (:1215-1475) and
    lm_loop (:1478-1527) under l_anel, on the polytropic background of
    magic_torch/radial_functions.py:70-165 (magic_b200.profiles.polytropic_background).

    radial loop  the anelastic nonlinear stage (Plan.nl_anel: the 18-19 grid
                 fields of the non-curl advection, get_nl_anel with viscous and
                 Ohmic heating, forward transforms, Courant), then mt_get_td with
                 the anelastic entropy finish (1/rho0) and the heating added to
                 the entropy's explicit term (step_time.py:1452-1455);
    lm loop      entropy (kappa, beta + dLtemp0 + 2/r), toroidal velocity (with
                 the density and viscosity terms of update_z.py:40-47), then the
                 angular-momentum corrections of stress-free runs
                 (update_z.py:446-475, mt_correct_am), the poloidal velocity and
                 pressure with the anelastic (w, p) operators and, on Chebyshev
                 levels, the integral constraint of the l = 0 pressure
                 (update_wp.py:121-135, 416-421), magnetic field when l_mag.

    Defaults are the reference's anelastic benchmark setup (configs/
    hydro_bench_anel_modal.yaml): 5 density scale heights, polytropic index
    2, gravity ~ 1/r^2, no magnetic field, stress-free boundaries with both
    angular-momentum corrections, Chebyshev levels (standard (w, p) form).
    The reference factorises the anelastic (w, p) matrices with LU
    (update_wp.py:239-352); this step applies the inverse of the same scaled
    matrices (the two agree to 2e-14 at 33 levels, 1.7e-11 at 129)."""

    def __init__(self, l_max, n_r, ek=1e-4, ra=3e6, pr=1.0, prmag=5.0, dt=1e-6, strat=5.0,
                 polind=2.0, g0=0.0, g1=0.0, g2=1.0, l_mag=False, ktopv=1, kbotv=1,
                 l_correct_AMz=True, l_correct_AMe=True, precision="fp64", radratio=0.35,
                 radial_scheme="chebyshev", fd_order=4, fd_order_bound=2, device=None,
                 cache=None, minc=1):
        self.l_mag = bool(l_mag)
        self.l_anel = True
        self._anel = dict(strat=float(strat), polind=float(polind), g0=float(g0),
                          g1=float(g1), g2=float(g2))
        super().__init__(l_max, n_r, ek=ek, ra=ra, pr=pr, prmag=prmag, dt=dt,
                         precision=precision, radratio=radratio, fd_order=fd_order,
                         fd_order_bound=fd_order_bound, ktopv=ktopv, kbotv=kbotv, device=device,
                         cache=cache, minc=minc, radial_scheme=radial_scheme)
        self.ViscHeatFac = float(self._bg["ViscHeatFac"])
        self.OhmLossFac = float(self._bg["OhmLossFac"])
        if l_correct_AMz or l_correct_AMe:
            hp = self.hprof
            prof = I.am_profiles(hp["r"], hp["rho0"], hp["beta"], hp["dbeta"], self.sch.rint)
            t = lambda x: torch.as_tensor(np.asarray(x, dtype=np.float64),
                                          device=self.device).contiguous()
            self.am = dict({k: t(v) for k, v in prof.items() if k != "c_moi_oc"},
                           rint=t(self.sch.rint), r=t(hp["r"]), c_moi_oc=prof["c_moi_oc"],
                           am_start=0.0, axial=bool(l_correct_AMz),
                           equatorial=bool(l_correct_AMe))

    def _background_key(self):
        return ("anel",) + tuple(self._anel.values())

    def _background(self, r, radratio, ek, ra, pr, prmag):
        from .profiles import polytropic_background

        self._bg = polytropic_background(r, radratio, pr=pr, ra=ra, ek=ek, prmag=prmag,
                                         l_mag=self.l_mag, **self._anel)
        return {k: self._bg[k] for k in ("rgrav", "rho0", "beta", "dbeta", "ddbeta", "dLtemp0",
                                         "orho1", "orho2", "otemp1")}

    def _p0_constraint(self):
        return I.p0_integral_constraint(self.sch, dict(self._bg, polind=self._anel["polind"]))

    def stage_outputs(self):
        return ("Advr", "Advt", "Advp", "VSr", "VSt") + (
            ("VxBr", "VxBt", "VxBp") if self.l_mag else ()) + ("heat",)

    @property
    def work(self):
        """Workspace of the fused (split or digit-split) anelastic stage; FP64 plans
        compose the stage from the FP64 kernels and need none (the plan reports 0
        where the digit-split stage composes too)."""
        if self._work is None:
            n = self.plan.nl_anel_workspace(self.n_r, self.l_mag, False) \
                if self.plan.precision in ("split", "ozaki") else 0
            self._work = torch.empty(max(int(n), 1), dtype=torch.uint8, device=self.device)
        return self._work

    def nonlinear_stage(self):
        f = self.f
        names = ("w", "dw", "ddw", "z", "dz", "s") + (
            ("b", "db", "ddb", "aj", "dj") if self.l_mag else ())
        _, dtr, dth = self.plan.nl_anel({k: f[k] for k in names}, self.prof, self.LFfac,
                                        self.ViscHeatFac, self.OhmLossFac, 2.5, 1.0, self.opm,
                                        l_mag=self.l_mag, out=self.nl_out, work=self.work)
        return dtr, dth
