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


def _inverse_ops(A, sch, zero_l0=False, identity_l0=False):
    """M_l = A_l^-1 through the reference's row scaling (1 / row max), the
    Chebyshev truncation and the DCT-I to grid values folded in; degree 0 zero or
    the identity where the reference's solve does that."""
    N = sch.n_r
    if zero_l0 or identity_l0:
        A = A.copy()
        A[0] = np.eye(N)
    fac = 1.0 / np.abs(A).max(axis=2)
    M = np.linalg.inv(fac[:, :, None] * A) * fac[:, None, :]
    if zero_l0:
        M[0] = 0.0
    if sch.chebyshev:
        M[:, sch.n_cheb:, :] = 0.0
        M = np.einsum("jk,lkn->ljn", _dct1(N), M)
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
    """Per-degree operator set on the GPU (mt_lop): one dense n_r x n_r matrix per l."""

    def __init__(self, M, device=None):
        M = np.ascontiguousarray(np.asarray(M, dtype=np.float64))
        if M.ndim != 3 or M.shape[1] != M.shape[2]:
            raise ValueError("expected (n_l, n_r, n_r) matrices")
        self.n_l, self.n_r = M.shape[0], M.shape[1]
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_lop_create(self.n_l, self.n_r,
                                           M.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h)))
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


def update_scalar(plan, sch, lop, s, ds, ta, weights, opr, hdif, kappa, d1c, or2, top=None,
                  bot=None):
    """One implicit entropy (or composition) step in place (magic_torch/update_s.py:213-271)."""
    update_field(plan, sch, lop, s, ds, ta, weights,
                 entropy_coefficients(plan.l_max, opr, hdif, np.asarray(kappa),
                                      np.asarray(d1c), np.asarray(or2)), top=top, bot=bot)
