"""Implicit field updates (CNAB2 right-hand side, per-degree solve, radial
derivatives, next implicit term, history rotation) on the GPU in FP64, for the
entropy, the toroidal velocity and the magnetic field: against the
reference's own updateS, updateZ and updateB outputs (tests/golden/td_*.npz) and against the numpy oracle for two
consecutive steps at l_max = 127 / 65 Chebyshev levels and l_max = 255 / 97
fourth-order finite-difference levels.

Tolerance 1e-12 relative to each array's largest value.  On Chebyshev and
second-order finite-difference levels the GPU applies the inverse of each
degree's matrix (with the DCT-I folded in for Chebyshev), as the reference
does there; on finite differences of order > 2 it solves with the pivoted
banded LU factors, in the reference's dgbsl order (the oracle restates the
same factorisation).  The implicit term is a second radial derivative of the
new field: at 65 Chebyshev levels ||D2||_inf ~ 1e7 amplifies rounding-level
differences, so it is held to 1e-11 (measured 1.9e-12).
"""

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err
from oracle import implicit as oi

pytestmark = pytest.mark.gpu

TOL = 1e-12
TOL_IMPL = 1e-11
cu = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()
npy = lambda t: t.cpu().numpy()


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
def test_update_scalar_matches_reference(name):
    from types import SimpleNamespace

    from magic_b200 import Plan
    from magic_b200 import implicit as I
    from magic_b200.radial import RadialOp

    z = load_golden(name)
    p = Plan(int(z["l_max"]), int(z["minc"]))
    sch = SimpleNamespace(n_r=int(z["n_r_max"]), chebyshev=bool(z["chebyshev"]),
                          n_cheb=int(z["n_cheb_max"]), rMat=z["rMat"], drMat=z["drMat"],
                          d2rMat=z["d2rMat"], rnorm=float(z["rnorm"]),
                          boundary_fac=float(z["boundary_fac"]), fd_order=int(z["fd_order"]),
                          D1=RadialOp(z["D1"]), D2=RadialOp(z["D2"]))
    d1c = z["beta"] + z["dLtemp0"] + 2 * z["or1"] + z["dLkappa"]
    w = I.cnab2_weights(1e-4, 1.3e-4)
    lop = I.LOp(I.scalar_solve_operators(sch, p.l_max, w[1], float(z["opr"]), z["hdif_S"],
                                         z["kappa"], d1c, z["or2"]))
    ta = {k: cu(z["s_" + k]) for k in ("old", "impl", "expl0", "expl1")}
    s = torch.empty_like(ta["old"])
    ds = torch.empty_like(ta["old"])
    I.update_scalar(p, sch, lop, s, ds, ta, w, float(z["opr"]), z["hdif_S"], z["kappa"], d1c,
                    z["or2"], top=cu(z["tops"]), bot=cu(z["bots"]))
    errs = dict(s=rel_err(npy(s), z["s_new"]), ds=rel_err(npy(ds), z["ds_new"]),
                impl=rel_err(npy(ta["impl"]), z["s_impl_new"]),
                old=rel_err(npy(ta["old"]), z["s_old_new"]),
                expl1=rel_err(npy(ta["expl1"]), z["s_expl1_new"]))
    print(name, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < TOL, (k, v)
    assert rel_err(npy(ta["expl0"]), z["s_expl0"]) == 0.0  # left for the next explicit stage


@pytest.mark.parametrize("scheme,l_max,n_r", [("chebyshev", 127, 65), ("FD", 255, 97),
                                               ("FD", 31, 289)])
def test_update_scalar_two_steps_vs_oracle(scheme, l_max, n_r):
    """Two consecutive steps against the oracle; 289 levels take the wide tiling
    (n_r > 256: solve matrices read from L2 instead of staged in shared memory)."""
    from magic_b200 import Plan
    from magic_b200 import implicit as I
    from magic_b200.radial import RadialScheme

    p = Plan(l_max, 1)
    fd = scheme == "FD"
    sch = RadialScheme(n_r, scheme, fd_order=4 if fd else 2)
    r = sch.r
    prof = dict(or1=1.0 / r, or2=1.0 / r ** 2, beta=-0.3 * np.ones(n_r) if fd else np.zeros(n_r),
                dLtemp0=-0.5 / r if fd else np.zeros(n_r), dLkappa=np.zeros(n_r),
                kappa=np.ones(n_r))
    d1c = prof["beta"] + prof["dLtemp0"] + 2 * prof["or1"] + prof["dLkappa"]
    hdif = np.ones(l_max + 1)
    opr = 1.0
    rng = np.random.default_rng(l_max)
    amp = (p.lm2l + 1.0)[:, None] ** -1.5
    spec = lambda: (rng.standard_normal((p.lm_max, n_r))
                    + 1j * rng.standard_normal((p.lm_max, n_r))) * amp
    st = dict(old=spec(), impl=spec(), expl0=spec(), expl1=spec())
    bots = np.zeros(p.lm_max, dtype=np.complex128)
    bots[0] = np.sqrt(4 * np.pi)
    tops = np.zeros_like(bots)
    ta = {k: cu(v) for k, v in st.items()}
    g = dict(lm2l=p.lm2l, lm2m=p.lm2m, l_max=l_max)
    mats = (sch.rMat, sch.drMat, sch.d2rMat, sch.rnorm, sch.boundary_fac)
    for step, (dt1, dt2) in enumerate(((2e-4, 2e-4), (1.5e-4, 2e-4))):
        w = I.cnab2_weights(dt1, dt2)
        lop = I.LOp(I.scalar_solve_operators(sch, l_max, w[1], opr, hdif, prof["kappa"], d1c,
                                             prof["or2"]))
        s = torch.empty_like(ta["old"])
        ds = torch.empty_like(ta["old"])
        I.update_scalar(p, sch, lop, s, ds, ta, w, opr, hdif, prof["kappa"], d1c, prof["or2"],
                        top=cu(tops), bot=cu(bots))
        ref = oi.update_s(g, mats, prof, st, ([w[0]], [w[1], w[2]], [w[3], w[4]]), opr, hdif,
                          tops, bots, sch.D1m, sch.D2m, sch.chebyshev, sch.n_cheb, sch.fd_order)
        for k, got in (("s", s), ("ds", ds), ("impl", ta["impl"]), ("old", ta["old"]),
                       ("expl1", ta["expl1"])):
            e = rel_err(npy(got), ref[k])
            assert e < (TOL_IMPL if k == "impl" else TOL), (scheme, step, k, e)
        # next step: the explicit stage would write a new expl0
        st = dict(old=ref["old"], impl=ref["impl"], expl0=spec(), expl1=ref["expl1"])
        ta["expl0"] = cu(st["expl0"])


def _sch_from(z):
    from types import SimpleNamespace

    from magic_b200.radial import RadialOp

    return SimpleNamespace(n_r=int(z["n_r_max"]), chebyshev=bool(z["chebyshev"]),
                           n_cheb=int(z["n_cheb_max"]), rMat=z["rMat"], drMat=z["drMat"],
                           d2rMat=z["d2rMat"], rnorm=float(z["rnorm"]),
                           boundary_fac=float(z["boundary_fac"]), fd_order=int(z["fd_order"]),
                           D1=RadialOp(z["D1"]), D2=RadialOp(z["D2"]))


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
def test_update_toroidal_matches_reference(name):
    from magic_b200 import Plan
    from magic_b200 import implicit as I

    z = load_golden(name)
    p = Plan(int(z["l_max"]), int(z["minc"]))
    sch = _sch_from(z)
    w = I.cnab2_weights(1e-4, 1.3e-4)
    args = (z["hdif_V"], z["visc"], z["beta"], z["dbeta"], z["dLvisc"], z["or1"], z["or2"])
    lop = I.LOp(I.toroidal_solve_operators(sch, p.l_max, w[1], *args, ktopv=int(z["ktopv"]),
                                           kbotv=int(z["kbotv"])))
    ta = {k: cu(z["z_" + k]) for k in ("old", "impl", "expl0", "expl1")}
    x, dx = torch.empty_like(ta["old"]), torch.empty_like(ta["old"])
    I.update_field(p, sch, lop, x, dx, ta, w, I.toroidal_coefficients(p.l_max, *args))
    errs = dict(z=rel_err(npy(x), z["z_new"]), dz=rel_err(npy(dx), z["dz_new"]),
                impl=rel_err(npy(ta["impl"]), z["z_impl_new"]),
                old=rel_err(npy(ta["old"]), z["z_old_new"]),
                expl1=rel_err(npy(ta["expl1"]), z["z_expl1_new"]))
    print(name, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < TOL, (k, v)


@pytest.mark.parametrize("scheme,l_max,n_r,k", [("chebyshev", 127, 65, 1), ("FD", 255, 97, 2)])
def test_update_toroidal_vs_oracle(scheme, l_max, n_r, k):
    from magic_b200 import Plan
    from magic_b200 import implicit as I
    from magic_b200.radial import RadialScheme

    p = Plan(l_max, 1)
    fd = scheme == "FD"
    sch = RadialScheme(n_r, scheme, fd_order=4 if fd else 2)
    r = sch.r
    prof = dict(or1=1.0 / r, or2=1.0 / r ** 2, beta=-0.3 / r if fd else np.zeros(n_r),
                dbeta=0.3 / r ** 2 if fd else np.zeros(n_r), dLvisc=np.zeros(n_r),
                visc=np.ones(n_r))
    hdif = np.ones(l_max + 1)
    rng = np.random.default_rng(7 * l_max)
    amp = (p.lm2l + 1.0)[:, None] ** -1.5
    st = {kk: (rng.standard_normal((p.lm_max, n_r)) + 1j * rng.standard_normal((p.lm_max, n_r)))
          * amp for kk in ("old", "impl", "expl0", "expl1")}
    ta = {kk: cu(v) for kk, v in st.items()}
    w = I.cnab2_weights(1e-4, 1.2e-4)
    args = (hdif, prof["visc"], prof["beta"], prof["dbeta"], prof["dLvisc"], prof["or1"],
            prof["or2"])
    lop = I.LOp(I.toroidal_solve_operators(sch, l_max, w[1], *args, ktopv=k, kbotv=k))
    x, dx = torch.empty_like(ta["old"]), torch.empty_like(ta["old"])
    I.update_field(p, sch, lop, x, dx, ta, w, I.toroidal_coefficients(l_max, *args))
    g = dict(lm2l=p.lm2l, lm2m=p.lm2m, l_max=l_max)
    mats = (sch.rMat, sch.drMat, sch.d2rMat, sch.rnorm, sch.boundary_fac)
    ref = oi.update_z(g, mats, prof, st, ([w[0]], [w[1], w[2]], [w[3], w[4]]), hdif, sch.D1m,
                      sch.D2m, sch.chebyshev, sch.n_cheb, k, k, sch.fd_order)
    for kk, got in (("x", x), ("dx", dx), ("impl", ta["impl"]), ("old", ta["old"]),
                    ("expl1", ta["expl1"])):
        e = rel_err(npy(got), ref[kk])
        assert e < (TOL_IMPL if kk == "impl" else TOL), (scheme, kk, e)


@pytest.mark.parametrize("name", ["td_cheb", "td_fd_anel"])
def test_update_magnetic_matches_reference(name):
    from magic_b200 import Plan
    from magic_b200 import implicit as I

    z = load_golden(name)
    p = Plan(int(z["l_max"]), int(z["minc"]))
    sch = _sch_from(z)
    w = I.cnab2_weights(1e-4, 1.3e-4)
    Mb, Mj = I.magnetic_solve_operators(sch, p.l_max, w[1], float(z["opm"]), z["hdif_B"],
                                        z["lambda_"], z["dLlambda"], z["or1"], z["or2"])
    cb, cj = I.magnetic_coefficients(p.l_max, float(z["opm"]), z["hdif_B"], z["lambda_"],
                                     z["dLlambda"], z["or2"])
    for f, M, c in (("b", Mb, cb), ("j", Mj, cj)):
        ta = {k: cu(z[f + "_" + k]) for k in ("old", "impl", "expl0", "expl1")}
        x, dx, d2x = (torch.empty_like(ta["old"]) for _ in range(3))
        I.update_field(p, sch, I.LOp(M), x, dx, ta, w, c, d2x=d2x)
        errs = dict(x=rel_err(npy(x), z[f + "_new"]), dx=rel_err(npy(dx), z["d" + f + "_new"]),
                    d2x=rel_err(npy(d2x), z["dd" + f + "_new"]),
                    impl=rel_err(npy(ta["impl"]), z[f + "_impl_new"]),
                    old=rel_err(npy(ta["old"]), z[f + "_old_new"]),
                    expl1=rel_err(npy(ta["expl1"]), z[f + "_expl1_new"]))
        print(name, f, {k: f"{v:.1e}" for k, v in errs.items()})
        for k, v in errs.items():
            assert v < TOL, (f, k, v)


@pytest.mark.parametrize("scheme,l_max,n_r", [("chebyshev", 127, 65), ("FD", 255, 97)])
def test_update_magnetic_vs_oracle(scheme, l_max, n_r):
    from magic_b200 import Plan
    from magic_b200 import implicit as I
    from magic_b200.radial import RadialScheme

    p = Plan(l_max, 1)
    fd = scheme == "FD"
    sch = RadialScheme(n_r, scheme, fd_order=4 if fd else 2)
    r = sch.r
    prof = dict(or1=1.0 / r, or2=1.0 / r ** 2, lambda_=np.ones(n_r),
                dLlambda=0.2 / r if fd else np.zeros(n_r))
    hdif, opm = np.ones(l_max + 1), 0.2
    rng = np.random.default_rng(11 * l_max)
    amp = (p.lm2l + 1.0)[:, None] ** -1.5
    spec = lambda: (rng.standard_normal((p.lm_max, n_r))
                    + 1j * rng.standard_normal((p.lm_max, n_r))) * amp
    st = {f: {k: spec() for k in ("old", "impl", "expl0", "expl1")} for f in ("b", "j")}
    w = I.cnab2_weights(1e-4, 1.2e-4)
    Mb, Mj = I.magnetic_solve_operators(sch, l_max, w[1], opm, hdif, prof["lambda_"],
                                        prof["dLlambda"], prof["or1"], prof["or2"])
    cb, cj = I.magnetic_coefficients(l_max, opm, hdif, prof["lambda_"], prof["dLlambda"],
                                     prof["or2"])
    g = dict(lm2l=p.lm2l, lm2m=p.lm2m, l_max=l_max)
    mats = (sch.rMat, sch.drMat, sch.d2rMat, sch.rnorm, sch.boundary_fac)
    ref = oi.update_b(g, mats, prof, st["b"], st["j"], ([w[0]], [w[1], w[2]], [w[3], w[4]]),
                      opm, hdif, sch.D1m, sch.D2m, sch.chebyshev, sch.n_cheb, sch.fd_order)
    for f, M, c, o in (("b", Mb, cb, ref[0]), ("j", Mj, cj, ref[1])):
        ta = {k: cu(v) for k, v in st[f].items()}
        x, dx, d2x = (torch.empty_like(ta["old"]) for _ in range(3))
        I.update_field(p, sch, I.LOp(M), x, dx, ta, w, c, d2x=d2x)
        for k, got in (("x", x), ("dx", dx), ("d2x", d2x), ("impl", ta["impl"]),
                       ("old", ta["old"]), ("expl1", ta["expl1"])):
            e = rel_err(npy(got), o[k])
            assert e < (TOL_IMPL if k in ("impl", "d2x") else TOL), (scheme, f, k, e)


WPROF = ("or1", "or2", "beta", "dbeta", "ddbeta", "visc", "dLvisc", "ddLvisc", "orho1", "rgrav",
         "rho0")


def _run_poloidal(p, sch, st, s_new, prof, hdif, BuoFac, w):
    from magic_b200 import implicit as I
    from magic_b200.radial import RadialOp

    lop = I.LOp(I.poloidal_dc_solve_operators(sch, p.l_max, w[1], hdif, prof))
    P0 = RadialOp(I.p0_inverse(sch, prof["beta"]))
    ta = {k: cu(v) for k, v in st.items()}
    x, dx, d2x, pr = (torch.zeros_like(ta["old"]) for _ in range(4))
    I.update_poloidal_dc(p, sch, lop, P0, x, dx, d2x, pr, ta, w, cu(s_new), prof, hdif, BuoFac)
    return dict(x=x, dx=dx, d2x=d2x, impl=ta["impl"], old=ta["old"], expl1=ta["expl1"],
                p0=pr[0].real)


def test_update_poloidal_matches_reference():
    from types import SimpleNamespace

    from magic_b200 import Plan
    from magic_b200 import implicit as I
    from magic_b200.radial import RadialOp

    z = load_golden("td_fd_anel")
    p = Plan(int(z["l_max"]), int(z["minc"]))
    sch = SimpleNamespace(n_r=int(z["n_r_max"]), chebyshev=False, D1m=z["drMat"],
                          D2m=z["d2rMat"], D3m=z["d3rMat"], D4m=z["d4rMat"], r=z["r"],
                          fd_order=int(z["fd_order"]), D1=RadialOp(z["D1"]), D2=RadialOp(z["D2"]))
    prof = {k: z[k] for k in WPROF}
    st = {k: z["w_" + k] for k in ("old", "impl", "expl0", "expl1")}
    o = _run_poloidal(p, sch, st, z["s_new"], prof, z["hdif_V"], float(z["BuoFac"]),
                      I.cnab2_weights(1e-4, 1.3e-4))
    errs = {k: rel_err(npy(o[k]), z[ref]) for k, ref in (
        ("x", "w_new"), ("dx", "dw_new"), ("d2x", "ddw_new"), ("impl", "w_impl_new"),
        ("old", "w_old_new"), ("expl1", "w_expl1_new"), ("p0", "p0_new"))}
    print({k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < TOL, (k, v)


@pytest.mark.parametrize("l_max,n_r,scale", [(255, 97, 1.0), (16, 129, 1.0), (16, 261, 1.0)])
def test_update_poloidal_vs_oracle(l_max, n_r, scale):
    """l_max = 255, 97 fourth-order finite-difference levels, anelastic-like
    profiles; and l_max = 16 at 261 levels, the wide tiling (n_r > 256).  GPU
    and oracle both solve the fourth-order double-curl operator with its pivoted
    banded LU factors (the reference's algorithm on these grids), so they agree
    to 1e-12 (1e-11 for the terms with D2 of the new field; at 261 levels the
    finest spacing amplifies the rounding of x in dx, d2x and the implicit term,
    bounds below);
    the dense inverse the GPU applied before differed from the factorised solve
    by 2.6e-12 at 97 levels and 8e-11 at 261 (conditioning ~ n_r^4)."""
    from magic_b200 import Plan
    from magic_b200 import implicit as I
    from magic_b200.radial import RadialScheme

    p = Plan(l_max, 1)
    sch = RadialScheme(n_r, "FD", fd_order=4)
    r = sch.r
    prof = dict(or1=1.0 / r, or2=1.0 / r ** 2, beta=-0.3 / r, dbeta=0.3 / r ** 2,
                ddbeta=-0.6 / r ** 3, visc=np.ones(n_r), dLvisc=np.zeros(n_r),
                ddLvisc=np.zeros(n_r), orho1=np.exp(-0.3 * (r[0] - r)), rgrav=r / r[0],
                rho0=np.exp(0.3 * (r[0] - r)))
    hdif, BuoFac = np.ones(l_max + 1), 1e3
    rng = np.random.default_rng(3)
    amp = (p.lm2l + 1.0)[:, None] ** -1.5
    spec = lambda: (rng.standard_normal((p.lm_max, n_r))
                    + 1j * rng.standard_normal((p.lm_max, n_r))) * amp
    st = {k: spec() for k in ("old", "impl", "expl0", "expl1")}
    s_new = spec()
    w = I.cnab2_weights(1e-4, 1.2e-4)
    o = _run_poloidal(p, sch, st, s_new, prof, hdif, BuoFac, w)
    g = dict(lm2l=p.lm2l, lm2m=p.lm2m, l_max=l_max)
    mats = (np.eye(n_r), sch.D1m, sch.D2m, sch.D3m, sch.D4m)
    ref = oi.update_w(g, mats, prof, st, ([w[0]], [w[1], w[2]], [w[3], w[4]]), hdif, sch.D1m,
                      sch.D2m, s_new, BuoFac, r, 4, 2, 2)
    errs = {k: rel_err(npy(o[k]), ref[k]) for k in ("x", "dx", "d2x", "impl", "old", "expl1",
                                                     "p0")}
    print(n_r, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, e in errs.items():
        if n_r > 256:
            # the finest spacing of 261 stretched levels: D1 and D2 (D4 in the
            # implicit term) of x amplify its rounding (measured x 2.8e-13,
            # dx 7.2e-12, d2x 2.9e-11, impl 8.3e-11, old 4.4e-12)
            tol = {"dx": 1e-11, "d2x": 1e-10, "impl": 1e-9, "old": 1e-10}.get(k, TOL)
        else:
            tol = TOL_IMPL if k in ("impl", "old", "d2x") else TOL
        assert e < scale * tol, (k, e)


WPPROF = ("or1", "or2", "beta", "dbeta", "visc", "dLvisc", "rgrav", "rho0")


def _run_wp(p, sch, stw, stp, s_new, prof, hdif, BuoFac, w, ktopv, kbotv):
    from magic_b200 import implicit as I
    from magic_b200.radial import RadialOp

    lop = I.LOp(I.wp_solve_operators(sch, p.l_max, w[1], hdif, prof, ktopv, kbotv))
    P0 = RadialOp(I.p0_inverse(sch, prof["beta"]))
    taw = {k: cu(v) for k, v in stw.items()}
    tap = {k: cu(v) for k, v in stp.items()}
    shape = taw["old"].shape
    out = {k: torch.full(shape, float("nan"), dtype=torch.complex128, device="cuda")
           for k in ("w", "dw", "ddw", "p", "dp")}
    I.update_wp(p, sch, lop, P0, out["w"], out["dw"], out["ddw"], out["p"], out["dp"], taw, tap,
                w, cu(s_new), prof, hdif, BuoFac)
    torch.cuda.synchronize()
    res = {k: npy(v) for k, v in out.items()}
    for f, ta in (("w", taw), ("p", tap)):
        for k in ("old", "impl", "expl0", "expl1"):
            res[f"{f}_{k}"] = npy(ta[k])
    return res


def test_update_wp_matches_reference():
    """The standard-form coupled (w, p) update with the l = 0 pressure
    (mt_update_wp) against the reference's own updateWP (tests/golden/td_cheb.npz:
    l_max 8, 9 Chebyshev levels, stress-free rows): w, dw, ddw, p, dp and both
    equations' old, implicit and rotated explicit terms.  The GPU applies the
    inverse of the scaled coupled matrix with the DCT-I folded in (the reference
    also applies a precomputed inverse, then the DCT-I)."""
    from types import SimpleNamespace

    from magic_b200 import Plan
    from magic_b200 import implicit as I
    from magic_b200.radial import RadialOp

    z = load_golden("td_cheb")
    p = Plan(int(z["l_max"]), int(z["minc"]))
    sch = SimpleNamespace(n_r=int(z["n_r_max"]), chebyshev=True, n_cheb=int(z["n_cheb_max"]),
                          rMat=z["rMat"], drMat=z["drMat"], d2rMat=z["d2rMat"],
                          d3rMat=z["d3rMat"], rnorm=float(z["rnorm"]),
                          boundary_fac=float(z["boundary_fac"]), D1=RadialOp(z["D1"]),
                          D2=RadialOp(z["D2"]), D3=RadialOp(z["D3"]))
    prof = {k: z[k] for k in WPPROF}
    stw = {k: z["wp_w_" + k] for k in ("old", "impl", "expl0", "expl1")}
    stp = {k: z["wp_p_" + k] for k in ("old", "impl", "expl0", "expl1")}
    o = _run_wp(p, sch, stw, stp, z["s_new"], prof, z["hdif_V"], float(z["BuoFac"]),
                I.cnab2_weights(1e-4, 1.3e-4), int(z["ktopv"]), int(z["kbotv"]))
    errs = {k: rel_err(o[k], z[f"wp_{k}_new"]) for k in ("w", "dw", "ddw", "p", "dp")}
    for f in ("w", "p"):
        for k in ("old", "impl", "expl1"):
            errs[f"{f}_{k}"] = rel_err(o[f"{f}_{k}"], z[f"wp_{f}_{k}_new"])
        assert rel_err(o[f"{f}_expl0"], z[f"wp_{f}_expl0"]) == 0.0
    print({k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < (TOL_IMPL if k in ("ddw", "p_impl", "w_impl", "dw") else TOL), (k, v)


@pytest.mark.parametrize("l_max,minc,n_r,ktopv,scale", [(127, 1, 65, 2, 1.0), (32, 4, 33, 1, 1.0),
                                                         (16, 1, 129, 2, 1e2),
                                                         (8, 1, 193, 2, 3e3)])
def test_update_wp_vs_oracle(l_max, minc, n_r, ktopv, scale):
    """l_max = 127 on 65 Chebyshev levels (no-slip) and l_max = 32, minc = 4 on 33
    levels (stress-free) with anelastic-like profiles, against the oracle's LU
    solves (the tensor-pipe tiling with four n-tiles per warp, n_r <= 128);
    l_max = 16 on 129 levels takes the six-tile variant (n_r <= 192, the
    anelastic benchmark's levels), l_max = 8 on 193 levels the FMA tiling.  The
    coupled Chebyshev operator is far worse conditioned than the scalar ones (its
    p rows carry d3rMat): the tolerances are relative to each array's largest
    value, 1e-11 for the fields and 1e-10 for the terms that apply D2 / D3 to the
    new w, scaled by 100 at 129 levels and 3000 at 193 (the conditioning grows
    ~ n_r^4 and the D3 norm ~ n_r^6; measured at 129 levels: fields <= 5.0e-12,
    ddw 6.9e-10, p_impl 3.4e-9; at 193: fields <= 2.7e-11, ddw 4.8e-9, p_impl
    7.7e-8)."""
    from magic_b200 import Plan
    from magic_b200 import implicit as I
    from magic_b200.radial import RadialScheme

    p = Plan(l_max, minc)
    sch = RadialScheme(n_r, "chebyshev")
    r = sch.r
    prof = dict(or1=1.0 / r, or2=1.0 / r ** 2, beta=-0.3 / r, dbeta=0.3 / r ** 2,
                visc=1.0 + 0.1 * r / r[0], dLvisc=0.1 / (r[0] + 0.1 * r), rgrav=r / r[0],
                rho0=np.exp(0.3 * (r[0] - r)))
    hdif, BuoFac = np.ones(l_max + 1), 1e3
    rng = np.random.default_rng(5)
    amp = (p.lm2l + 1.0)[:, None] ** -1.5
    spec = lambda: (rng.standard_normal((p.lm_max, n_r))
                    + 1j * rng.standard_normal((p.lm_max, n_r))) * amp
    stw = {k: spec() for k in ("old", "impl", "expl0", "expl1")}
    stp = {k: spec() for k in ("old", "impl", "expl0", "expl1")}
    s_new = spec()
    w = I.cnab2_weights(1e-4, 1.2e-4)
    o = _run_wp(p, sch, stw, stp, s_new, prof, hdif, BuoFac, w, ktopv, ktopv)
    g = dict(lm2l=p.lm2l, lm2m=p.lm2m, l_max=l_max)
    mats = (sch.rMat, sch.drMat, sch.d2rMat, sch.rnorm, sch.boundary_fac)
    ref = oi.update_wp(g, mats, sch.d3rMat, prof, {k: v.copy() for k, v in stw.items()},
                       {k: v.copy() for k, v in stp.items()},
                       ([w[0]], [w[1], w[2]], [w[3], w[4]]), hdif, sch.D1m, sch.D2m, sch.D3m,
                       s_new, BuoFac, sch.n_cheb, ktopv, ktopv)
    errs = {k: rel_err(o[k], ref[k]) for k in ("w", "dw", "ddw", "p", "dp", "w_old", "w_impl",
                                                "w_expl1", "p_old", "p_impl", "p_expl1")}
    print({k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < scale * (1e-10 if k in ("ddw", "w_impl", "p_impl", "p_old", "dw", "dp")
                            else 1e-11), (k, v)
