"""Implicit (IMEX) updates on the GPU: CNAB2 weights, per-degree solve
operators (built once per time step size on the host, as the reference builds
and factorises its matrices) and the scalar-field update
(magic_torch/update_s.py:67-271; update_xi.py has the same form).

Layout of the time arrays: one contiguous (lm_max, n_r) complex128 tensor per
time level (``old``, ``impl``, ``expl0``, ``expl1``), instead of the
reference's (lm_max, n_r, n_levels) TimeArray; the update rotates the
explicit history itself (expl1 <- expl0) and stores the new field as ``old``.
"""

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from ._lib import check


def cnab2_weights(dt1, dt2, alpha=0.6):
    """(w_old, w_impl_now, w_impl_prev, w_expl0, w_expl1) of CNAB2 with time steps
    dt1 (current) and dt2 (previous) (magic_torch/time_scheme.py:56-73):
    wimp = 1, wimp_lin = (alpha dt1, (1 - alpha) dt1), wexp = ((1 + dt1/(2 dt2)) dt1,
    -dt1^2/(2 dt2)).  w_impl_now multiplies the implicit operator in the matrices."""
    return (1.0, alpha * dt1, (1.0 - alpha) * dt1, (1.0 + 0.5 * dt1 / dt2) * dt1,
            -0.5 * dt1 * dt1 / dt2)


def _dct1(n):
    N = n - 1
    k = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    Cm = 2.0 * np.cos(np.pi * ((j * k) % (2 * N)) / N)
    Cm[:, 0] = 1.0
    Cm[:, N] = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    return Cm / np.sqrt(2.0 * N)


class Band:
    """Preconditioned per-degree LHS for a pivoted banded LU solve: A (n_l, n_r,
    n_r) with kl sub- and ku super-diagonals, the row scaling fr (n_l, n_r) and
    the column scaling fc (or None) of the solve x = fc U^-1 L^-1 P (fr rhs)."""

    def __init__(self, A, fr, fc, kl, ku):
        self.A, self.fr, self.fc, self.kl, self.ku = A, fr, fc, int(kl), int(ku)


def _banded(sch):
    """The reference factorises instead of inverting on finite-difference grids of
    order > 2 (magic_torch/update_s.py:95-104 and the same test in update_z.py,
    update_b.py, update_w_doublecurl.py)."""
    return (not sch.chebyshev) and getattr(sch, "fd_order", 2) > 2


def _band_width(sch):
    """kl = ku of the S, Z, B and J matrices on such grids: max(fd_order / 2,
    fd_order_bound) (update_s.py:101, update_z.py:125, update_b.py:129)."""
    return max(sch.fd_order // 2, getattr(sch, "fd_order_bound", 2))


def _inverse_ops(A, sch, zero_l0=False, identity_l0=False):
    """M_l = A_l^-1 through the reference's row scaling (1 / row max), the
    Chebyshev truncation and the DCT-I to grid values folded in; degree 0 zero or
    the identity where the reference's solve does that.  On finite-difference
    grids of order > 2 the row-scaled matrices are returned for a banded LU
    solve instead (Band)."""
    N = sch.n_r
    if _banded(sch):
        A = A.copy()
        if zero_l0 or identity_l0:
            A[0] = np.eye(N)
        fac = 1.0 / np.abs(A).max(axis=2)
        kl = _band_width(sch)
        return Band(fac[:, :, None] * A, fac, None, kl, kl)
    if zero_l0 or identity_l0:
        A = A.copy()
        A[0] = np.eye(N)
    fac = 1.0 / np.abs(A).max(axis=2)
    M = np.linalg.inv(fac[:, :, None] * A) * fac[:, None, :]
    if zero_l0:
        M[0] = 0.0
    if sch.chebyshev:
        M[:, sch.n_cheb:, :] = 0.0
        M = np.matmul(_dct1(N)[None], M)
    return M


def _bc_rows(A, sch, rows):
    """Boundary rows (row index -> matrix row, or one row per degree), the
    Chebyshev columns >= n_cheb dropped in them, then columns 0 and n_r-1 scaled
    by boundary_fac."""
    N = sch.n_r
    for i, v in rows.items():
        A[:, i, :] = v
    if sch.n_cheb < N:
        A[:, 0, sch.n_cheb:] = 0.0
        A[:, N - 1, sch.n_cheb:] = 0.0
    A[:, :, 0] *= sch.boundary_fac
    A[:, :, N - 1] *= sch.boundary_fac
    return A


def scalar_solve_operators(sch, l_max, wimp_lin0, opr, hdif, kappa, d1c, or2):
    """(l_max+1, n_r, n_r) solve operators M_l of the entropy / composition LHS
    (magic_torch/update_s.py:67-134):
        A_l = rnorm (rMat - wimp_lin0 opr hdif_l kappa (d2rMat + d1c drMat
              - l(l+1) or2 rMat)),
    Dirichlet rows 0 and n_r-1 (rnorm rMat)."""
    ls = np.arange(l_max + 1, dtype=np.float64)
    dL = (ls * (ls + 1.0))[:, None, None]
    op = sch.d2rMat[None] + d1c[None, :, None] * sch.drMat[None] - dL * or2[None, :, None] * sch.rMat[None]
    A = sch.rnorm * (sch.rMat[None] - wimp_lin0 * opr * np.asarray(hdif)[:, None, None]
                     * kappa[None, :, None] * op)
    N = sch.n_r
    A = _bc_rows(A, sch, {0: sch.rnorm * sch.rMat[0], N - 1: sch.rnorm * sch.rMat[N - 1]})
    return _inverse_ops(A, sch)


def toroidal_solve_operators(sch, l_max, wimp_lin0, hdif, visc, beta, dbeta, dLvisc, or1, or2,
                             ktopv=2, kbotv=2):
    """(l_max+1, n_r, n_r) solve operators of the toroidal-velocity LHS
    (magic_torch/update_z.py:89-240):
        A_l = rnorm l(l+1) or2 (rMat - wimp_lin0 hdif_l visc (d2rMat + (dLvisc - beta) drMat
              - (dLvisc beta + 2 dLvisc or1 + l(l+1) or2 + dbeta + 2 beta or1) rMat)),
    boundary rows stress-free (k = 1: rnorm (drMat - (2 or1 + beta) rMat)) or no-slip
    (rnorm rMat).  Degree 0: zero, except the identity of the banded finite-difference
    solve (fd_order > 2)."""
    N = sch.n_r
    ls = np.arange(l_max + 1, dtype=np.float64)
    dL = (ls * (ls + 1.0))[:, None, None]
    c0 = (dLvisc * beta + 2.0 * dLvisc * or1)[None, :, None] + dL * or2[None, :, None] \
        + (dbeta + 2.0 * beta * or1)[None, :, None]
    op = sch.d2rMat[None] + (dLvisc - beta)[None, :, None] * sch.drMat[None] - c0 * sch.rMat[None]
    A = sch.rnorm * dL * or2[None, :, None] * (
        sch.rMat[None] - wimp_lin0 * np.asarray(hdif)[:, None, None] * visc[None, :, None] * op)
    rows = {}
    for i, k in ((0, ktopv), (N - 1, kbotv)):
        rows[i] = (sch.rnorm * (sch.drMat[i] - (2.0 * or1[i] + beta[i]) * sch.rMat[i]) if k == 1
                   else sch.rnorm * sch.rMat[i])
    A = _bc_rows(A, sch, rows)
    banded_l0 = (not sch.chebyshev) and getattr(sch, "fd_order", 2) > 2
    return _inverse_ops(A, sch, zero_l0=not banded_l0, identity_l0=banded_l0)


def magnetic_solve_operators(sch, l_max, wimp_lin0, opm, hdif, lam, dLlam, or1, or2):
    """(M_b, M_j): solve operators of the poloidal and toroidal magnetic field with
    an insulating inner core and mantle (magic_torch/update_b.py:98-280):
        bulk rows  rnorm l(l+1) or2 (rMat - wimp_lin0 opm lambda hdif_l (d2rMat
                   [+ dLlambda drMat for j] - l(l+1) or2 rMat)),
        b: rows rnorm (drMat + l or1 rMat) at the top and rnorm (drMat - (l+1) or1 rMat)
           at the bottom (potential-field matching), j: Dirichlet rows rnorm rMat.
    Degree 0: zero, except the identity of the banded finite-difference solve."""
    N = sch.n_r
    ls = np.arange(l_max + 1, dtype=np.float64)
    dL = (ls * (ls + 1.0))[:, None, None]
    hd = np.asarray(hdif, dtype=np.float64)[:, None, None]
    base = sch.rnorm * dL * or2[None, :, None]
    lap = dL * or2[None, :, None] * sch.rMat[None]
    Ab = base * (sch.rMat[None] - wimp_lin0 * opm * lam[None, :, None] * hd
                 * (sch.d2rMat[None] - lap))
    Aj = base * (sch.rMat[None] - wimp_lin0 * opm * lam[None, :, None] * hd
                 * (sch.d2rMat[None] + dLlam[None, :, None] * sch.drMat[None] - lap))
    top = sch.rnorm * (sch.drMat[0][None] + ls[:, None] * or1[0] * sch.rMat[0][None])
    bot = sch.rnorm * (sch.drMat[N - 1][None] - (ls[:, None] + 1.0) * or1[N - 1]
                       * sch.rMat[N - 1][None])
    Ab = _bc_rows(Ab, sch, {0: top, N - 1: bot})
    Aj = _bc_rows(Aj, sch, {0: sch.rnorm * sch.rMat[0], N - 1: sch.rnorm * sch.rMat[N - 1]})
    banded_l0 = (not sch.chebyshev) and getattr(sch, "fd_order", 2) > 2
    return (_inverse_ops(Ab, sch, zero_l0=not banded_l0, identity_l0=banded_l0),
            _inverse_ops(Aj, sch, zero_l0=not banded_l0, identity_l0=banded_l0))


def magnetic_coefficients(l_max, opm, hdif, lam, dLlam, or2):
    """Coefficients of mt_update_field for b and j (magic_torch/update_b.py:616-631):
    old = l(l+1) or2 x; impl = opm lambda hdif l(l+1) or2 (d2x [+ dLlambda dx for j]
    - l(l+1) or2 x)."""
    ls = np.arange(l_max + 1, dtype=np.float64)
    dLh = ls * (ls + 1.0)
    ia_l = opm * np.asarray(hdif, dtype=np.float64) * dLh
    common = dict(so_l=dLh, so_r=or2, ia_l=ia_l, ia_r=lam * or2, ic_r=None, ic_l=dLh, ic_r2=or2)
    return dict(common, ib_r=np.zeros_like(or2)), dict(common, ib_r=dLlam)


def _w_coefficient_profiles(prof):
    """(c3, c2n, c1n, c1d, c0n) of the double-curl diffusion operator
    (magic_torch/update_w_doublecurl.py:146-168): c2 = c2n - 2 l(l+1) or2,
    c1 = c1n + l(l+1) c1d, c0 = l(l+1) or2 (c0n + l(l+1) or2)."""
    dLv, ddLv, b, db, ddb, or1, or2 = (prof[k] for k in ("dLvisc", "ddLvisc", "beta", "dbeta",
                                                          "ddbeta", "or1", "or2"))
    c3 = 2.0 * (dLv - b)
    c2n = ddLv - 2.0 * db + dLv ** 2 + b ** 2 - 3.0 * dLv * b - 2.0 * or1 * (dLv + b)
    c1n = (-ddb - db * (2.0 * dLv - b + 2.0 * or1) - ddLv * (b + 2.0 * or1)
           + b ** 2 * (dLv + 2.0 * or1) - b * (dLv ** 2 - 2.0 * or2)
           - 2.0 * dLv * or1 * (dLv - or1))
    c1d = 2.0 * (2.0 * or1 + b - dLv) * or2
    c0n = (2.0 * db + ddLv + dLv ** 2 - (2.0 / 3.0) * b ** 2 + dLv * b
           + 2.0 * or1 * (2.0 * dLv - b - 3.0 * or1))
    return c3, c2n, c1n, c1d, c0n


def poloidal_dc_solve_operators(sch, l_max, wimp_lin0, hdif, prof, ktopv=2, kbotv=2):
    """(l_max+1, n_r, n_r) solve operators of the double-curl poloidal LHS on
    finite-difference grid values (magic_torch/update_w_doublecurl.py:67-300):
    rows 2..n_r-3  -l(l+1) or2 orho1 (d2 - beta d - l(l+1) or2)
                   + wimp_lin0 orho1 hdif_l visc l(l+1) or2 (d4 + c3 d3 + c2 d2 + c1 d + c0),
    rows 0, n_r-1: w = 0; rows 1, n_r-2: dw = 0 (no-slip) or d2w - (2 or1 + beta) dw = 0
    (stress-free) at the boundary.  Inverted through the reference's row, then column
    scaling; degree 0 zero.  prof: or1, or2, beta, dbeta, ddbeta, visc, dLvisc,
    ddLvisc, orho1 over n_r."""
    if sch.chebyshev:
        raise ValueError("the double-curl form is used with finite differences only")
    N = sch.n_r
    D = (np.eye(N), sch.D1m, sch.D2m, sch.D3m, sch.D4m)
    c3, c2n, c1n, c1d, c0n = _w_coefficient_profiles(prof)
    or1, or2, beta, orho1, visc = (prof[k] for k in ("or1", "or2", "beta", "orho1", "visc"))
    banded = _banded(sch)
    M = np.zeros((l_max + 1, N, N))
    if banded:  # degree 0: the identity (update_w_doublecurl.py:136-139)
        M[0] = np.eye(N)
        FR, FC = np.ones((l_max + 1, N)), np.ones((l_max + 1, N))
    b = slice(2, N - 2)
    for l in range(1, l_max + 1):
        dL = float(l * (l + 1))
        dLo = dL * or2
        old = (-dLo * orho1)[b, None] * (D[2][b] - beta[b, None] * D[1][b] - dLo[b, None] * D[0][b])
        c2, c1, c0 = c2n - 2.0 * dLo, c1n + dL * c1d, dLo * (c0n + dLo)
        imp = (orho1 * hdif[l] * visc * dLo)[b, None] * (
            D[4][b] + c3[b, None] * D[3][b] + c2[b, None] * D[2][b] + c1[b, None] * D[1][b]
            + c0[b, None] * D[0][b])
        A = np.zeros((N, N))
        A[b] = old + wimp_lin0 * imp
        A[0], A[N - 1] = D[0][0], D[0][N - 1]
        A[1] = (D[2][0] - (2.0 * or1[0] + beta[0]) * D[1][0]) if ktopv == 1 else D[1][0]
        A[N - 2] = ((D[2][N - 1] - (2.0 * or1[N - 1] + beta[N - 1]) * D[1][N - 1])
                    if kbotv == 1 else D[1][N - 1])
        fr = 1.0 / np.abs(A).max(axis=1)
        A = fr[:, None] * A
        fc = 1.0 / np.abs(A).max(axis=0)
        if banded:
            M[l], FR[l], FC[l] = A * fc[None, :], fr, fc
        else:
            M[l] = fc[:, None] * np.linalg.inv(A * fc[None, :]) * fr[None, :]
    if banded:
        # n_bands = max(fd_order + 3, 2 fd_order_bound + 3) (update_w_doublecurl.py:111-117)
        kl = (max(sch.fd_order + 3, 2 * getattr(sch, "fd_order_bound", 2) + 3) - 1) // 2
        return Band(M, FR, FC, kl, kl)
    return M


def wp_solve_operators(sch, l_max, wimp_lin0, hdif, prof, ktopv=2, kbotv=2):
    """(l_max+1, 2 n_r, 2 n_r) solve operators of the coupled (w, p) LHS of the
    standard poloidal form on Chebyshev levels (magic_torch/update_wp.py:197-368,
    get_wpMat): unknowns the Chebyshev coefficients of w (0..n_r-1) and p
    (n_r..2n_r-1),
      w rows 1..n_r-2  rnorm l(l+1) or2 (rMat - wimp hdif_l visc (d2rMat
                       + (2 dLvisc - beta/3) drMat - (l(l+1) or2 + 4/3 (dLvisc beta
                       + (3 dLvisc + beta) or1 + dbeta)) rMat))  |  rnorm wimp (drMat - beta rMat)
      p rows           rnorm l(l+1) or2 (-drMat - wimp hdif_l visc (-d3rMat
                       + (beta - dLvisc) d2rMat + (l(l+1) or2 + dbeta + dLvisc beta
                       + 2 (dLvisc + beta) or1) drMat - l(l+1) or2 (2 or1 + dLvisc
                       + 2/3 beta) rMat))  |  -rnorm wimp l(l+1) or2 rMat
      boundary rows    w = 0 at both ends; dw = 0 (no-slip) or d2w - (2 or1 + beta) dw
                       = 0 (stress-free) in rows n_r, 2n_r-1,
    Chebyshev columns >= n_cheb dropped in the boundary rows, the first and last
    column of each block scaled by boundary_fac; inverted through the reference's
    row, then column scaling; the Chebyshev truncation and the DCT-I of each block
    folded in, so the operators map the right-hand side to grid values; degree 0
    zero.  prof: or1, or2, beta, dbeta, visc, dLvisc over n_r."""
    if not sch.chebyshev:
        raise ValueError("the standard (w, p) form is used with the Chebyshev scheme only")
    N, nc = sch.n_r, sch.n_cheb
    rMat, drMat, d2rMat, d3rMat, rn = sch.rMat, sch.drMat, sch.d2rMat, sch.d3rMat, sch.rnorm
    col = lambda k: np.asarray(prof[k], dtype=np.float64)[:, None]
    or1, or2, beta, dbeta, visc, dLv = (col(k) for k in ("or1", "or2", "beta", "dbeta", "visc",
                                                         "dLvisc"))
    b = slice(1, N - 1)
    C2 = np.zeros((2 * N, 2 * N))
    C2[:N, :N] = C2[N:, N:] = _dct1(N)
    # every degree at once: (l_max, 2N, 2N) for l = 1 .. l_max, broadcast over l
    ls = np.arange(1, l_max + 1, dtype=np.float64)
    dL = (ls * (ls + 1.0))[:, None, None]
    hl = np.asarray(hdif, dtype=np.float64)[1:l_max + 1, None, None]
    A = np.zeros((l_max, 2 * N, 2 * N))
    A[:, b, :N] = rn * dL * or2[b] * (rMat[b] - wimp_lin0 * hl * visc[b] * (
        d2rMat[b] + (2.0 * dLv[b] - beta[b] / 3.0) * drMat[b]
        - (dL * or2[b] + 4.0 / 3.0 * (dLv[b] * beta[b] + (3.0 * dLv[b] + beta[b]) * or1[b]
                                      + dbeta[b])) * rMat[b]))
    A[:, b, N:] = rn * wimp_lin0 * (drMat[b] - beta[b] * rMat[b])
    A[:, N + 1:2 * N - 1, :N] = rn * dL * or2[b] * (-drMat[b] - wimp_lin0 * hl * visc[b] * (
        -d3rMat[b] + (beta[b] - dLv[b]) * d2rMat[b]
        + (dL * or2[b] + dbeta[b] + dLv[b] * beta[b] + 2.0 * (dLv[b] + beta[b]) * or1[b])
        * drMat[b]
        - dL * or2[b] * (2.0 * or1[b] + dLv[b] + 2.0 / 3.0 * beta[b]) * rMat[b]))
    A[:, N + 1:2 * N - 1, N:] = -rn * wimp_lin0 * dL * or2[b] * rMat[b]
    A[:, 0, :N], A[:, N - 1, :N] = rn * rMat[0], rn * rMat[N - 1]
    for row, i, k in ((N, 0, ktopv), (2 * N - 1, N - 1, kbotv)):
        A[:, row, :N] = rn * ((d2rMat[i] - (2.0 * or1[i, 0] + beta[i, 0]) * drMat[i]) if k == 1
                              else drMat[i])
    if nc < N:
        for row in (0, N - 1, N, 2 * N - 1):
            A[:, row, nc:N] = 0.0
            A[:, row, N + nc:] = 0.0
    for c in (0, N - 1, N, 2 * N - 1):
        A[:, :, c] *= sch.boundary_fac
    fr = 1.0 / np.abs(A).max(axis=2)
    A = fr[:, :, None] * A
    fc = 1.0 / np.abs(A).max(axis=1)
    Minv = fc[:, :, None] * np.linalg.inv(A * fc[:, None, :]) * fr[:, None, :]
    if nc < N:
        Minv[:, nc:N] = 0.0
        Minv[:, N + nc:] = 0.0
    M = np.zeros((l_max + 1, 2 * N, 2 * N))
    M[1:] = np.matmul(C2[None], Minv)
    return M


def cheb_integral_kernel(N, rnorm):
    """K[j, k] = rnorm (1/(1 - (k-j)^2) + 1/(1 - (k+j)^2)) / 2 for j + k even (terms
    with a zero denominator dropped), else 0: the integral of T_j T_k over [-1, 1]
    in the reference's Chebyshev normalisation (magic_torch/init_fields.py:88-105)."""
    j = np.arange(N, dtype=np.float64)[:, None]
    k = np.arange(N, dtype=np.float64)[None, :]
    d1, d2 = 1.0 - (k - j) ** 2, 1.0 - (k + j) ** 2
    with np.errstate(divide="ignore"):
        s1 = np.where(d1 != 0, 1.0 / np.where(d1 != 0, d1, 1.0), 0.0)
        s2 = np.where(d2 != 0, 1.0 / np.where(d2 != 0, d2, 1.0), 0.0)
    return ((j + k) % 2 == 0) * (s1 + s2) * 0.5 * rnorm


def p0_integral_constraint(sch, bg, ThExpNb=1.0):
    """The anelastic l = 0 pressure's integral constraint on Chebyshev levels
    (magic_torch/update_wp.py:31, 121-135, 416-421; used when ViscHeatFac ThExpNb
    != 0): (row, rhs) with row the physical weights ThExpNb ViscHeatFac ogrun
    alpha0 r^2 whose Chebyshev integral replaces the p = 0 row of the matrix
    (ogrun = polind, alpha0 = 1 / temp0), and rhs the weights of the right-hand
    side's row 0, int ThExpNb alpha0 temp0 rho0 r^2 Re s00 dr = sum rhs Re s00
    (radial rule sch.rint).  None where the constraint is off (Boussinesq, or FD)."""
    if not sch.chebyshev or bg["ViscHeatFac"] * ThExpNb == 0.0:
        return None
    r = np.asarray(sch.r, dtype=np.float64)
    alpha0, temp0, rho0 = 1.0 / bg["temp0"], bg["temp0"], bg["rho0"]
    ogrun = np.full_like(r, bg["polind"])
    row = ThExpNb * bg["ViscHeatFac"] * ogrun * alpha0 * r * r
    rhs = np.asarray(sch.rint) * ThExpNb * alpha0 * temp0 * rho0 * r * r
    return row, rhs


def _lapack_inverse(A):
    """FP64 inverse by torch.linalg.inv on the CPU, the routine the reference uses
    for its l = 0 pressure matrix (magic_torch/update_wp.py:141-171)."""
    return torch.linalg.inv(torch.from_numpy(np.ascontiguousarray(A, dtype=np.float64))).numpy()


def p0_inverse(sch, beta, integ_row=None):
    """Inverse of the l = 0 pressure matrix (magic_torch/update_wp.py:80-165).
    Finite differences: grid-value unknowns, rows 1.. dp/dr - beta p with the last
    row the first-order backward difference (entries beyond the band of half-width
    fd_order/2 dropped), row 0 p = 0.  Chebyshev: coefficient unknowns, rows rnorm
    (drMat - beta rMat); row 0 rnorm rMat[0] (p = 0 at the outer boundary) or, with
    integ_row (p0_integral_constraint), the Chebyshev integral of integ_row p: K
    applied to rnorm costf(integ_row) with its end values times boundary_fac;
    columns >= n_cheb dropped in row 0, first and last column scaled by
    boundary_fac, with the truncation and the DCT-I to grid values folded into
    the inverse.  Inverted with the reference's own routine (torch.linalg.inv on
    the CPU): with the integral row the matrix's condition number reaches ~5e8,
    and two LAPACK inversions then differ by ~1e-10 in the hydrostatic p00,
    while the same routine reproduces the reference's inverse exactly."""
    N = sch.n_r
    if sch.chebyshev:
        A = np.zeros((N, N))
        A[1:] = sch.rnorm * (sch.drMat[1:] - np.asarray(beta)[1:, None] * sch.rMat[1:])
        if integ_row is not None:
            work = _dct1(N) @ np.asarray(integ_row, dtype=np.float64) * sch.rnorm
            work[0] *= sch.boundary_fac
            work[N - 1] *= sch.boundary_fac
            A[0] = cheb_integral_kernel(N, sch.rnorm) @ work
        else:
            A[0] = sch.rnorm * sch.rMat[0]
        if sch.n_cheb < N:
            A[0, sch.n_cheb:] = 0.0
        A[:, 0] *= sch.boundary_fac
        A[:, N - 1] *= sch.boundary_fac
        Minv = _lapack_inverse(A)
        Minv[sch.n_cheb:] = 0.0
        return _dct1(N) @ Minv
    A = np.zeros((N, N))
    A[1:] = sch.D1m[1:] - beta[1:, None] * np.eye(N)[1:]
    delr = sch.r[N - 1] - sch.r[N - 2]
    A[N - 1, N - 1] = 1.0 / delr - beta[N - 1]
    A[N - 1, N - 2] = -1.0 / delr
    A[N - 1, :N - 1 - sch.fd_order // 2] = 0.0
    A[0] = np.eye(N)[0]
    return _lapack_inverse(A)


def update_poloidal_dc(plan, sch, lop, P0, w, dw, ddw, p, ta, weights, s, prof, hdif, BuoFac,
                       xi=None, ChemFac=0.0, wcoef=None):
    """One double-curl poloidal step in place (mt_update_poloidal): w, dw, ddw outputs,
    p (row (0, 0) written: the l = 0 pressure), ta: dict old, impl, expl0, expl1;
    s / xi: this step's entropy / composition; prof: or1, or2, beta, dbeta, ddbeta,
    visc, dLvisc, ddLvisc, orho1, rgrav, rho0 over n_r (numpy or device arrays);
    P0: RadialOp of p0_inverse; wcoef: precomputed _w_coefficient_profiles(prof)."""
    n_r = w.shape[1]
    arrs = [w, dw, ddw, ta["old"], ta["impl"], ta["expl0"], ta["expl1"], p, s]
    for a in arrs + ([xi] if xi is not None else []):
        if a.shape != w.shape or a.dtype != torch.complex128 or not a.is_contiguous():
            raise ValueError("fields and time arrays must be contiguous (lm_max, n_r) complex128")
    w_old, wimp_lin0, w_impl, w_e0, w_e1 = weights
    c3, c2n, c1n, c1d, c0n = wcoef if wcoef is not None else _w_coefficient_profiles(prof)
    prof_arrays = [hdif] + [prof[k] for k in (
        "or2", "orho1", "beta", "visc", "rgrav", "rho0")] + [c3, c2n, c1n, c1d, c0n]
    dev = [torch.as_tensor(v, dtype=torch.float64, device=w.device).contiguous()
           for v in prof_arrays]
    u = _lib.PoloidalUpdate(*[a.data_ptr() for a in arrs],
                            xi.data_ptr() if xi is not None else None, n_r,
                            w_old, w_impl, w_e0, w_e1, wimp_lin0, float(BuoFac), float(ChemFac),
                            *[d.data_ptr() for d in dev])
    st = C.c_void_p(torch.cuda.current_stream(w.device).cuda_stream)
    check(_lib.lib().mt_update_poloidal(plan._h, n_r, C.byref(u), lop._h, sch.D1._h, sch.D2._h,
                                        P0._h, st))


def update_wp(plan, sch, lop, P0, w, dw, ddw, p, dp, taw, tap, weights, s, prof, hdif,
              BuoFac, xi=None, ChemFac=0.0, impl_interior=False, p0_row0=None):
    """One standard-form poloidal step in place (mt_update_wp): w, dw, ddw, p, dp
    outputs; taw / tap: dicts old, impl, expl0, expl1 of the w and p equations;
    s / xi: this step's entropy / composition; prof: or1, or2, beta, dbeta, visc,
    dLvisc, rgrav, rho0 over n_r (numpy or device arrays); lop: LOp of
    wp_solve_operators; P0: RadialOp of p0_inverse.  impl_interior: zero both
    implicit terms at l = 0 and at the boundary levels, as the reference's time
    step does (step_time.py:385-394; updateWP alone keeps them; the solution
    never reads those entries).  p0_row0: the anelastic integral constraint's
    right-hand-side weights (p0_integral_constraint), with P0 built from the same
    constraint; None: p = 0 at the outer boundary."""
    n_r = w.shape[1]
    arrs = [w, dw, ddw, p, dp, taw["old"], taw["impl"], taw["expl0"], taw["expl1"], tap["old"],
            tap["impl"], tap["expl0"], tap["expl1"], s]
    for a in arrs + ([xi] if xi is not None else []):
        if a.shape != w.shape or a.dtype != torch.complex128 or not a.is_contiguous():
            raise ValueError("fields and time arrays must be contiguous (lm_max, n_r) complex128")
    w_old, wimp_lin0, w_impl, w_e0, w_e1 = weights
    dev = [torch.as_tensor(v, dtype=torch.float64, device=w.device).contiguous()
           for v in [hdif] + [prof[k] for k in ("or1", "or2", "beta", "dbeta", "visc", "dLvisc",
                                               "rgrav", "rho0")]]
    u = _lib.WpUpdate(*[a.data_ptr() for a in arrs], xi.data_ptr() if xi is not None else None,
                      n_r, w_old, w_impl, w_e0, w_e1, wimp_lin0, float(BuoFac), float(ChemFac),
                      *[d.data_ptr() for d in dev], int(bool(impl_interior)),
                      p0_row0.data_ptr() if p0_row0 is not None else None)
    st = C.c_void_p(torch.cuda.current_stream(w.device).cuda_stream)
    check(_lib.lib().mt_update_wp(plan._h, n_r, C.byref(u), lop._h, sch.D1._h, sch.D2._h,
                                  sch.D3._h, P0._h, st))


def entropy_coefficients(l_max, opr, hdif, kappa, d1c, or2):
    """Coefficients of mt_update_field for entropy / composition
    (magic_torch/update_s.py:262-270): old = s, impl = opr hdif kappa
    (d2s + d1c ds - l(l+1) or2 s)."""
    ls = np.arange(l_max + 1, dtype=np.float64)
    return dict(so_l=None, so_r=None, ia_l=opr * np.asarray(hdif, dtype=np.float64), ia_r=kappa,
                ib_r=d1c, ic_r=None, ic_l=ls * (ls + 1.0), ic_r2=or2)


def toroidal_coefficients(l_max, hdif, visc, beta, dbeta, dLvisc, or1, or2):
    """Coefficients of mt_update_field for the toroidal velocity
    (magic_torch/update_z.py:37-47, 481-495): old = l(l+1) or2 z, impl = hdif l(l+1)
    or2 visc (d2z + (dLvisc - beta) dz - (dLvisc beta + 2 dLvisc or1 + dbeta
    + 2 beta or1 + l(l+1) or2) z)."""
    ls = np.arange(l_max + 1, dtype=np.float64)
    dLh = ls * (ls + 1.0)
    return dict(so_l=dLh, so_r=or2, ia_l=np.asarray(hdif, dtype=np.float64) * dLh,
                ia_r=or2 * visc, ib_r=dLvisc - beta,
                ic_r=dLvisc * beta + 2.0 * dLvisc * or1 + dbeta + 2.0 * beta * or1,
                ic_l=dLh, ic_r2=or2)


class LOp:
    """Per-degree operator set on the GPU (mt_lop): one dense n_r x n_r matrix per l
    (an inverse, applied as a product), or a Band (pivoted banded LU factors,
    solved in the reference's order)."""

    def __init__(self, M, device=None):
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        h = C.c_void_p()
        if isinstance(M, Band):
            A = np.ascontiguousarray(np.asarray(M.A, dtype=np.float64))
            fr = np.ascontiguousarray(np.asarray(M.fr, dtype=np.float64))
            fc = (np.ascontiguousarray(np.asarray(M.fc, dtype=np.float64)) if M.fc is not None
                  else None)
            self.n_l, self.n_r = A.shape[0], A.shape[1]
            self.banded = True
            with torch.cuda.device(self.device):
                check(_lib.lib().mt_lop_create_band(self.n_l, self.n_r, M.kl, M.ku, dp(A), dp(fr),
                                                    dp(fc) if fc is not None else None,
                                                    C.byref(h)))
            self._h = h
            return
        M = np.ascontiguousarray(np.asarray(M, dtype=np.float64))
        if M.ndim != 3 or M.shape[1] != M.shape[2]:
            raise ValueError("expected (n_l, n_r, n_r) matrices")
        self.n_l, self.n_r = M.shape[0], M.shape[1]
        self.banded = False
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_lop_create(self.n_l, self.n_r, dp(M), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().mt_lop_destroy(h)
            except Exception:
                pass
            self._h = None


def update_field(plan, sch, lop, x, dx, ta, weights, coef, top=None, bot=None, d2x=None):
    """One implicit step of a field in place (mt_update_field): x, dx (and d2x when
    given) (lm_max, n_r) complex128 outputs; ta: dict old, impl, expl0, expl1 of the
    same shape (updated in place); weights: cnab2_weights(...); coef:
    entropy_coefficients(...), toroidal_coefficients(...) or one of
    magnetic_coefficients(...); top / bot: (lm_max) complex boundary values or None."""
    n_r = x.shape[1]
    arrs = [x, dx, ta["old"], ta["impl"], ta["expl0"], ta["expl1"]]
    for a in arrs:
        if a.shape != x.shape or a.dtype != torch.complex128 or not a.is_contiguous():
            raise ValueError("fields and time arrays must be contiguous (lm_max, n_r) complex128")
    w_old, _, w_impl, w_e0, w_e1 = weights
    names = ("so_l", "so_r", "ia_l", "ia_r", "ib_r", "ic_r", "ic_l", "ic_r2")
    dev = {k: (torch.as_tensor(coef[k], dtype=torch.float64, device=x.device).contiguous()
               if coef.get(k) is not None else None) for k in names}
    if d2x is not None and (d2x.shape != x.shape or d2x.dtype != torch.complex128
                            or not d2x.is_contiguous()):
        raise ValueError("d2x must be a contiguous (lm_max, n_r) complex128 array")
    u = _lib.FieldUpdate(arrs[0].data_ptr(), arrs[1].data_ptr(),
                         d2x.data_ptr() if d2x is not None else None,
                         *[a.data_ptr() for a in arrs[2:]],
                         top.data_ptr() if top is not None else None,
                         bot.data_ptr() if bot is not None else None, n_r,
                         w_old, w_impl, w_e0, w_e1,
                         *[dev[k].data_ptr() if dev[k] is not None else None for k in names])
    st = C.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)
    check(_lib.lib().mt_update_field(plan._h, n_r, C.byref(u), lop._h, sch.D1._h, sch.D2._h, st))


def am_profiles(r, rho0, beta, dbeta, rint):
    """Profiles of the angular-momentum corrections (magic_torch/update_z.py:57-64):
    am_z = rho0 r^2, am_dz = rho0 (2 r + r^2 beta), am_d2z = rho0 (2 + 4 beta r
    + (dbeta + beta^2) r^2), and the outer core's moment of inertia c_moi_oc =
    8/3 pi int r^4 rho0 dr (pre_calculations.py:94-98) with the radial rule rint."""
    r, rho0, beta, dbeta, rint = (np.asarray(x, dtype=np.float64)
                                  for x in (r, rho0, beta, dbeta, rint))
    r2 = r * r
    return dict(am_z=rho0 * r2, am_dz=rho0 * (2.0 * r + r2 * beta),
                am_d2z=rho0 * (2.0 + 4.0 * beta * r + dbeta * r2 + beta * beta * r2),
                c_moi_oc=8.0 / 3.0 * math.pi * float(np.dot(rint, r2 * r2 * rho0)))


def correct_am(plan, z, dz, ta, coef, am, d2z=None):
    """The angular-momentum corrections after the toroidal update (mt_correct_am,
    magic_torch/update_z.py:446-475): z, dz (d2z) and the old / implicit terms in
    ta of the rows (l, m) = (1, 0) and (1, 1), in place.  coef: the toroidal
    coefficients the update used; am: device profiles rint, r, am_z, am_dz, am_d2z
    (am_profiles) and c_moi_oc, am_start, axial, equatorial."""
    n_r = z.shape[1]
    names = ("so_l", "so_r", "ia_l", "ia_r", "ib_r", "ic_r", "ic_l", "ic_r2")
    ptr = lambda x: x.data_ptr() if x is not None else None
    for a in (z, dz, ta["old"], ta["impl"]):
        if a.shape != z.shape or a.dtype != torch.complex128 or not a.is_contiguous():
            raise ValueError("fields and time arrays must be contiguous (lm_max, n_r) complex128")
    u = _lib.FieldUpdate(z.data_ptr(), dz.data_ptr(), ptr(d2z), ta["old"].data_ptr(),
                         ta["impl"].data_ptr(), None, None, None, None, n_r, 0.0, 0.0, 0.0, 0.0,
                         *[ptr(coef.get(k)) for k in names])
    c = _lib.AmCorrection(*[am[k].data_ptr() for k in ("rint", "r", "am_z", "am_dz", "am_d2z")],
                          float(am["c_moi_oc"]), float(am["am_start"]), int(am["axial"]),
                          int(am["equatorial"]))
    st = C.c_void_p(torch.cuda.current_stream(z.device).cuda_stream)
    check(_lib.lib().mt_correct_am(plan._h, n_r, C.byref(u), C.byref(c), st))


def update_scalar(plan, sch, lop, s, ds, ta, weights, opr, hdif, kappa, d1c, or2, top=None,
                  bot=None):
    """One implicit entropy (or composition) step in place (magic_torch/update_s.py:213-271)."""
    update_field(plan, sch, lop, s, ds, ta, weights,
                 entropy_coefficients(plan.l_max, opr, hdif, np.asarray(kappa),
                                      np.asarray(d1c), np.asarray(or2)), top=top, bot=bot)
