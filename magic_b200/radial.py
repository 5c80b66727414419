"""Radial schemes and radial operators on the GPU.

Host-side set-up, as in the reference (built once on the CPU in FP64):

* Chebyshev-Gauss-Lobatto grid and derivative matrices D_k = d^k rMat .
  rMat^-1 (magic_torch/chebyshev.py:21-120, radial_derivatives.py:71-100);
* finite-difference grid (uniform or stretched) and derivative matrices
  from Fornberg's weights (magic_torch/finite_differences.py:21-330).

The operators themselves run on the GPU through the C ABI
(``mt_radial_op_*``, ``mt_radial_apply``): ``get_dr``, ``get_ddr``,
``get_dddr`` and ``costf`` keep the signatures of
magic_torch/radial_derivatives.py:29-68 and cosine_transform.py:18-45,
with the operator passed explicitly instead of read from module state.
"""

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from ._lib import check

_CD = torch.complex128


# ---------------------------------------------------------------- Chebyshev

def cheb_grid(n_r, radratio=0.35):
    """r[k] = (r_cmb - r_icb)/2 cos(pi k / N) + (r_icb + r_cmb)/2, k = 0..N = n_r - 1,
    r_cmb = 1/(1 - radratio), r_icb = r_cmb - 1 (magic_torch/chebyshev.py:21-45)."""
    N = n_r - 1
    r_cmb = 1.0 / (1.0 - radratio)
    r_icb = r_cmb - 1.0
    x = np.cos(math.pi * np.arange(n_r, dtype=np.float64) / N)
    return 0.5 * (r_cmb - r_icb) * x + 0.5 * (r_icb + r_cmb), x


def cheb_polynomials(n_r, radratio=0.35, third=False):
    """(rMat, drMat, d2rMat): T_n(x_i) and its first two r-derivatives at the
    Gauss-Lobatto points (magic_torch/chebyshev.py:62-110); with third=True also
    d3rMat, the third derivatives."""
    _, x = cheb_grid(n_r, radratio)
    r_cmb = 1.0 / (1.0 - radratio)
    drx = 2.0 / (r_cmb - (r_cmb - 1.0))
    T = np.zeros((n_r, n_r))
    dT = np.zeros((n_r, n_r))
    d2T = np.zeros((n_r, n_r))
    d3T = np.zeros((n_r, n_r))
    T[:, 0] = 1.0
    T[:, 1] = x
    dT[:, 1] = drx
    for c in range(2, n_r):
        T[:, c] = 2.0 * x * T[:, c - 1] - T[:, c - 2]
        dT[:, c] = 2.0 * drx * T[:, c - 1] + 2.0 * x * dT[:, c - 1] - dT[:, c - 2]
        d2T[:, c] = 4.0 * drx * dT[:, c - 1] + 2.0 * x * d2T[:, c - 1] - d2T[:, c - 2]
        d3T[:, c] = 6.0 * drx * d2T[:, c - 1] + 2.0 * x * d3T[:, c - 1] - d3T[:, c - 2]
    return (T, dT, d2T, d3T) if third else (T, dT, d2T)


def cheb_matrices(n_r, radratio=0.35, n_cheb=None):
    """(r, D1, D2, D3): D_k = d^k rMat . rMat^-1 with rMat[i, n] = T_n(x_i) and the
    derivative columns from the three-term recurrence with the linear map
    dx/dr = 2 / (r_cmb - r_icb); Chebyshev modes >= n_cheb are dropped
    (magic_torch/chebyshev.py:62-110, radial_derivatives.py:71-100)."""
    r, x = cheb_grid(n_r, radratio)
    r_cmb = 1.0 / (1.0 - radratio)
    drx = 2.0 / (r_cmb - (r_cmb - 1.0))
    T = np.zeros((n_r, n_r))
    dT = np.zeros((n_r, n_r))
    d2T = np.zeros((n_r, n_r))
    d3T = np.zeros((n_r, n_r))
    T[:, 0] = 1.0
    T[:, 1] = x
    dT[:, 1] = drx
    for c in range(2, n_r):
        T[:, c] = 2.0 * x * T[:, c - 1] - T[:, c - 2]
        dT[:, c] = 2.0 * drx * T[:, c - 1] + 2.0 * x * dT[:, c - 1] - dT[:, c - 2]
        d2T[:, c] = 4.0 * drx * dT[:, c - 1] + 2.0 * x * d2T[:, c - 1] - d2T[:, c - 2]
        d3T[:, c] = 6.0 * drx * d2T[:, c - 1] + 2.0 * x * d3T[:, c - 1] - d3T[:, c - 2]
    Tinv = np.linalg.inv(T)
    if n_cheb is not None and n_cheb < n_r:
        Tinv[n_cheb:, :] = 0.0
    return r, dT @ Tinv, d2T @ Tinv, d3T @ Tinv


# ------------------------------------------------------ finite differences

def fornberg_weights(z, x, m):
    """Weights c[j, k] of the k-th derivative at z from values at x[j], k <= m
    (B. Fornberg, Math. Comp. 51 (1988) 699-706; as used by
    magic_torch/finite_differences.py:21-58)."""
    nd = len(x) - 1
    c = np.zeros((nd + 1, m + 1))
    c1, c4 = 1.0, x[0] - z
    c[0, 0] = 1.0
    for i in range(1, nd + 1):
        mn = min(i, m)
        c2, c5, c4 = 1.0, c4, x[i] - z
        for j in range(i):
            c3 = x[i] - x[j]
            c2 *= c3
            if j == i - 1:
                for k in range(mn, 0, -1):
                    c[i, k] = c1 * (k * c[i - 1, k - 1] - c5 * c[i - 1, k]) / c2
                c[i, 0] = -c1 * c5 * c[i - 1, 0] / c2
            for k in range(mn, 0, -1):
                c[j, k] = (c4 * c[j, k] - k * c[j, k - 1]) / c3
            c[j, 0] = c4 * c[j, 0] / c3
        c1 = c2
    return c


def fd_grid(n_r, radratio=0.35, stretch=0.3, ratio=0.1):
    """Radial grid from r_cmb down to r_icb: uniform when ratio == 1, else fine
    boundary layers whose spacing grows geometrically (factor ratio^(-1/nb))
    into a uniform bulk (magic_torch/finite_differences.py:61-136)."""
    r_cmb = 1.0 / (1.0 - radratio)
    r_icb = r_cmb - 1.0
    r = np.zeros(n_r)
    r[0] = r_cmb
    if ratio == 1.0:
        for i in range(1, n_r):
            r[i] = r[i - 1] - 1.0 / (n_r - 1)
    else:
        nb = int((n_r - 1) / (2.0 * (1.0 + stretch)))
        full = abs(r_icb) <= 10.0 * np.finfo(np.float64).eps
        n_bulk = n_r - 1 - nb if full else n_r - 1 - 2 * nb
        g = math.exp(math.log(ratio) / nb)
        p = 1.0
        for _ in range(nb):
            p *= g
        h = 1.0 / (n_bulk + (1.0 if full else 2.0) * g * (1.0 - p) / (1.0 - g))
        for _ in range(nb):
            h *= g
        for i in range(1, nb + 1):
            r[i] = r[i - 1] - h
            h /= g
        for i in range(n_bulk):
            r[nb + 1 + i] = r[nb + i] - h
        if not full:
            for i in range(nb):
                h *= g
                r[nb + n_bulk + 1 + i] = r[nb + n_bulk + i] - h
    r[n_r - 1] = r_icb
    return r


def fd_matrices(r, order=2, order_boundary=2):
    """(D1, D2, D3, D4) dense finite-difference derivative matrices: centred
    order+1 point stencils in the bulk (order+3 for D3, D4), one-sided
    stencils of order_boundary at the ends; bottom rows mirror the top ones
    (magic_torch/finite_differences.py:139-330)."""
    n = len(r)
    h = order // 2
    D = [np.zeros((n, n)) for _ in range(4)]

    def w(idx, row, m):
        return fornberg_weights(0.0, np.array([r[k] - r[row] for k in idx]), m)

    if order == 2:
        for j in range(n):
            if j in (0, n - 1):
                continue
            c = w([j - 1, j, j + 1], j, 2)
            D[0][j, j - 1:j + 2] = c[:, 1]
            D[1][j, j - 1:j + 2] = c[:, 2]
        for j in range(2, n - 2):
            c = w(range(j - 2, j + 3), j, 4)
            D[2][j, j - 2:j + 3] = c[:, 3]
            D[3][j, j - 2:j + 3] = c[:, 4]
    else:
        for j in range(h, n - h):
            c = w(range(j - h, j + h + 1), j, order)
            D[0][j, j - h:j + h + 1] = c[:, 1]
            D[1][j, j - h:j + h + 1] = c[:, 2]
        for j in range(1 + h, n - h - 1):
            c = w(range(j - h - 1, j + h + 2), j, order + 2)
            D[2][j, j - h - 1:j + h + 2] = c[:, 3]
            D[3][j, j - h - 1:j + h + 2] = c[:, 4]
    ob = order_boundary
    for j in range(h):
        c = w(range(ob + 1), j, ob)
        D[0][j, :ob + 1] = c[:, 1]
        c = w([n - 1 - od for od in range(ob + 1)], n - 1 - j, ob)
        D[0][n - 1 - j, n - ob - 1:] = c[::-1, 1]
        c = w(range(ob + 2), j, ob + 1)
        D[1][j, :ob + 2] = c[:, 2]
        c = w([n - 1 - od for od in range(ob + 2)], n - 1 - j, ob + 1)
        D[1][n - 1 - j, n - ob - 2:] = c[::-1, 2]
    for j in range(h + 1):
        c = w(range(ob + 3), j, ob + 2)
        D[2][j, :ob + 3] = c[:, 3]
        c = w([n - 1 - od for od in range(ob + 3)], n - 1 - j, ob + 2)
        D[2][n - 1 - j, n - ob - 3:] = c[::-1, 3]
        c = w(range(ob + 4), j, 4)
        D[3][j, :ob + 4] = c[:, 4]
        c = w([n - 1 - od for od in range(ob + 4)], n - 1 - j, 4)
        D[3][n - 1 - j, n - ob - 4:] = c[::-1, 4]
    return tuple(D)


# ---------------------------------------------------------- GPU operators

class RadialOp:
    """A real n_r x n_r matrix applied along the radial axis on the GPU
    (mt_radial_op).  Built from a host matrix; only each row's nonzero band is
    kept, so finite-difference operators cost their band."""

    def __init__(self, D=None, n_r=None, kind="matrix", device=None):
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        L = _lib.lib()
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            if kind == "dct1":
                self.n_r = int(n_r)
                check(L.mt_radial_op_create_dct1(self.n_r, C.byref(h)))
            else:
                M = np.ascontiguousarray(np.asarray(D, dtype=np.float64))
                if M.ndim != 2 or M.shape[0] != M.shape[1]:
                    raise ValueError("radial operator must be a square matrix")
                self.n_r = M.shape[0]
                check(L.mt_radial_op_create(self.n_r, M.ctypes.data_as(C.POINTER(C.c_double)),
                                            C.byref(h)))
        self._h = h

    @property
    def bandwidth(self):
        return _lib.lib().mt_radial_op_bandwidth(self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().mt_radial_op_destroy(h)
            except Exception:
                pass
            self._h = None

    def _rows(self, f):
        if f.dtype != _CD or f.device != self.device or f.shape[-1] != self.n_r:
            raise ValueError(f"expected complex128 (..., {self.n_r}) on {self.device}")
        return f.contiguous()

    def __call__(self, f):
        f = self._rows(f)
        out = torch.empty_like(f)
        nrows = f.numel() // self.n_r
        st = C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        check(_lib.lib().mt_radial_apply(self._h, nrows, f.data_ptr(), self.n_r,
                                         out.data_ptr(), self.n_r, st))
        return out


def get_dr(f, D1):
    """First radial derivative (magic_torch/radial_derivatives.py:29-38)."""
    return D1(f)


def get_ddr(f, D1, D2):
    """First and second radial derivatives in one pass (radial_derivatives.py:41-54)."""
    f = D1._rows(f)
    d1, d2 = torch.empty_like(f), torch.empty_like(f)
    st = C.c_void_p(torch.cuda.current_stream(D1.device).cuda_stream)
    check(_lib.lib().mt_radial_apply2(D1._h, D2._h, f.numel() // D1.n_r, f.data_ptr(), D1.n_r,
                                      d1.data_ptr(), d2.data_ptr(), D1.n_r, st))
    return d1, d2


def get_dddr(f, D1, D2, D3):
    """First to third radial derivatives (radial_derivatives.py:57-68)."""
    d1, d2 = get_ddr(f, D1, D2)
    return d1, d2, D3(f)


def dct1_matrix(n_r):
    """The self-inverse DCT-I of cosine_transform.py:18-45 as an n_r x n_r matrix:
    y[k] = (f[0] + (-1)^k f[N] + 2 sum_{0<j<N} f[j] cos(pi j k / N)) / sqrt(2 N)."""
    N = n_r - 1
    k = np.arange(n_r)[:, None]
    j = np.arange(n_r)[None, :]
    C = 2.0 * np.cos(np.pi * j * k / N)
    C[:, 0] = 1.0
    C[:, N] = (-1.0) ** np.arange(n_r)
    return C / np.sqrt(2.0 * N)


def simpson_weights(r):
    """Weights of the non-uniform Simpson rule of magic_torch/integration.py:73-121
    (odd n_r: composite Simpson; even: the mean of the two Simpson sweeps closed by
    a trapezoid at either end), integral = sum_r w[r] f[r], sign for r[0] = r_cmb."""
    r = np.asarray(r, dtype=np.float64)
    N = r.size
    w = np.zeros(N)

    def simpson(start, acc):
        for n in range(start, N - 1, 2):
            h1, h2 = r[n] - r[n - 1], r[n + 1] - r[n]
            c = (h1 + h2) / 6.0
            acc[n - 1] += c * (2.0 * h1 - h2) / h1
            acc[n] += c * (h1 + h2) * (h1 + h2) / (h1 * h2)
            acc[n + 1] += c * (2.0 * h2 - h1) / h2

    if N % 2 == 1:
        simpson(1, w)
        return -w
    w[0] += 0.5 * (r[1] - r[0])
    w[1] += 0.5 * (r[1] - r[0])
    simpson(2, w)
    w[N - 1] += 0.5 * (r[N - 1] - r[N - 2])
    w[N - 2] += 0.5 * (r[N - 1] - r[N - 2])
    simpson(1, w)
    return -0.5 * w


def clenshaw_curtis_weights(n_r, radratio, rnorm, boundary_fac):
    """Weights of the Chebyshev integration of magic_torch/integration.py:18-70:
    DCT-I of f / drx (drx = 2 / (r_cmb - r_icb)), end coefficients times
    boundary_fac, dotted with the Chebyshev integrals (1 for T_0, -1/((n+1)(n-1))
    for even n > 0, 0 for odd n), times 2 rnorm."""
    r_cmb = 1.0 / (1.0 - radratio)
    r_icb = radratio / (1.0 - radratio)
    drx = 2.0 / (r_cmb - r_icb)
    ci = np.zeros(n_r)
    ci[0] = 1.0
    for n in range(2, n_r, 2):
        ci[n] = -1.0 / ((n + 1) * (n - 1))
    b = np.ones(n_r)
    b[0] = b[-1] = boundary_fac
    return 2.0 * rnorm / drx * ((ci * b) @ dct1_matrix(n_r))


_DCT = {}


def costf(f):
    """Self-inverse DCT-I along the last axis (magic_torch/cosine_transform.py:18-45)."""
    key = (f.shape[-1], f.device)
    if key not in _DCT:
        _DCT[key] = RadialOp(n_r=f.shape[-1], kind="dct1", device=f.device)
    return _DCT[key](f)


class RadialScheme:
    """Grid and derivative operators of one radial discretisation
    (magic_torch/radial_scheme.py): "chebyshev" or "FD"."""

    def __init__(self, n_r, scheme="chebyshev", radratio=0.35, n_cheb=None, fd_order=2,
                 fd_order_bound=2, fd_stretch=0.3, fd_ratio=0.1, device=None):
        self.n_r = n_r
        self.chebyshev = scheme.upper() != "FD"
        self.fd_order = fd_order
        self.fd_order_bound = fd_order_bound
        self.n_cheb = n_r if (n_cheb is None or not self.chebyshev) else min(n_cheb, n_r)
        if not self.chebyshev:
            self.r = fd_grid(n_r, radratio, fd_stretch, fd_ratio)
            allm = fd_matrices(self.r, fd_order, fd_order_bound)
            mats, self.D4m = allm[:3], allm[3]
            # grid-point unknowns: rMat = I, rnorm = boundary_fac = 1
            # (magic_torch/finite_differences.py:296-300)
            self.rMat, self.drMat, self.d2rMat = np.eye(n_r), mats[0], mats[1]
            self.rnorm, self.boundary_fac = 1.0, 1.0
        else:
            self.r, *mats = cheb_matrices(n_r, radratio, n_cheb)
            self.rMat, self.drMat, self.d2rMat, self.d3rMat = cheb_polynomials(n_r, radratio,
                                                                                third=True)
            # Chebyshev-coefficient unknowns (magic_torch/chebyshev.py:47-52)
            self.rnorm, self.boundary_fac = math.sqrt(2.0 / (n_r - 1)), 0.5
        self.radratio = radratio
        # radial integration rule as weights (magic_torch/integration.py:138)
        self.rint = (clenshaw_curtis_weights(n_r, radratio, self.rnorm, self.boundary_fac)
                     if self.chebyshev else simpson_weights(self.r))
        self.D1m, self.D2m, self.D3m = mats
        self.D1, self.D2, self.D3 = (RadialOp(M, device=device) for M in mats)
