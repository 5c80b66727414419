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


def scalar_solve_operators(sch, l_max, wimp_lin0, opr, hdif, kappa, d1c, or2):
    """(l_max+1, n_r, n_r) solve operators M_l of the scalar-field LHS
    (magic_torch/update_s.py:67-134):
        A_l = rnorm (rMat - wimp_lin0 opr hdif_l kappa (d2rMat + d1c drMat
              - l(l+1) or2 rMat)),
    Dirichlet rows 0 and n_r-1 (rnorm rMat, Chebyshev columns >= n_cheb dropped),
    columns 0 and n_r-1 scaled by boundary_fac; M_l = A_l^-1 through the same row
    scaling (1 / row max) the reference factorises with.  For the Chebyshev scheme
    the truncation to n_cheb modes and the DCT-I to grid values are folded in."""
    N = sch.n_r
    ls = np.arange(l_max + 1, dtype=np.float64)
    dL = (ls * (ls + 1.0))[:, None, None]
    op = sch.d2rMat[None] + d1c[None, :, None] * sch.drMat[None] - dL * or2[None, :, None] * sch.rMat[None]
    A = sch.rnorm * (sch.rMat[None] - wimp_lin0 * opr * np.asarray(hdif)[:, None, None]
                     * kappa[None, :, None] * op)
    A[:, 0, :] = sch.rnorm * sch.rMat[0, :]
    A[:, N - 1, :] = sch.rnorm * sch.rMat[N - 1, :]
    if sch.n_cheb < N:
        A[:, 0, sch.n_cheb:] = 0.0
        A[:, N - 1, sch.n_cheb:] = 0.0
    A[:, :, 0] *= sch.boundary_fac
    A[:, :, N - 1] *= sch.boundary_fac
    fac = 1.0 / np.abs(A).max(axis=2)
    M = np.linalg.inv(fac[:, :, None] * A) * fac[:, None, :]
    if sch.chebyshev:
        M[:, sch.n_cheb:, :] = 0.0
        M = np.einsum("jk,lkn->ljn", _dct1(N), M)
    return M


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


def update_scalar(plan, sch, lop, s, ds, ta, weights, opr, hdif, kappa, d1c, or2, top=None,
                  bot=None):
    """One implicit step of a scalar field in place (magic_torch/update_s.py:213-271).

    s, ds: (lm_max, n_r) complex128 outputs; ta: dict old, impl, expl0, expl1 of the
    same shape (updated in place); weights: cnab2_weights(...); hdif (l_max+1),
    kappa, d1c = beta + dLtemp0 + 2/r + dLkappa, or2 (n_r) real tensors on the device;
    top / bot: (lm_max) complex boundary values or None (zero)."""
    n_r = s.shape[1]
    arrs = [s, ds, ta["old"], ta["impl"], ta["expl0"], ta["expl1"]]
    for x in arrs:
        if x.shape != s.shape or x.dtype != torch.complex128 or not x.is_contiguous():
            raise ValueError("fields and time arrays must be contiguous (lm_max, n_r) complex128")
    w_old, _, w_impl, w_e0, w_e1 = weights
    prof = [torch.as_tensor(v, dtype=torch.float64, device=s.device).contiguous()
            for v in (hdif, kappa, d1c, or2)]
    u = _lib.ScalarUpdate(*[x.data_ptr() for x in arrs],
                          top.data_ptr() if top is not None else None,
                          bot.data_ptr() if bot is not None else None, n_r,
                          w_old, w_impl, w_e0, w_e1, float(opr), *[p.data_ptr() for p in prof])
    st = C.c_void_p(torch.cuda.current_stream(s.device).cuda_stream)
    check(_lib.lib().mt_update_scalar(plan._h, n_r, C.byref(u), lop._h, sch.D1._h, sch.D2._h,
                                      st))
