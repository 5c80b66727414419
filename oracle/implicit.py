"""CPU restatement (numpy, FP64) of the implicit update of a scalar field
(entropy; composition has the same form) with the CNAB2 scheme.  Test
infrastructure only: the library never imports this module.

Pinned against the reference's own updateS outputs (tests/golden/td_*.npz).
"""

import numpy as np

from oracle.td import dct1_matrix


def band_factor(A, kl, ku):
    """Pivoted banded LU of the dense matrix A (zero outside kl sub- and ku
    super-diagonals), in band storage abd[kl + ku + i - j, j] = A[i, j]: the
    reference's dense_to_band_storage and prepare_band (magic_torch/algebra.py:
    642-670, 371-457, a port of LINPACK dgbfa; 1-based indices as there).
    Returns (abd, pivot) with 1-based pivots."""
    n = A.shape[0]
    nb = 2 * kl + ku + 1
    abd = np.zeros((nb, n))
    for j in range(n):
        for i in range(max(0, j - ku), min(n, j + kl + 1)):
            abd[kl + ku + i - j, j] = A[i, j]
    m = kl + ku + 1
    piv = np.zeros(n, dtype=np.int64)
    a = lambda i, j: (i - 1, j - 1)
    for jz in range(ku + 2, min(n, m) - 1 + 1):
        for i in range(m + 1 - jz, kl + 1):
            abd[a(i, jz)] = 0.0
    jz, ju = min(n, m) - 1, 0
    for k in range(1, n):
        jz += 1
        if jz <= n:
            for i in range(1, kl + 1):
                abd[a(i, jz)] = 0.0
        lm = min(kl, n - k)
        col = np.abs(abd[m - 1:m + lm, k - 1])
        l = int(np.argmax(col)) + m
        piv[k - 1] = l + k - m
        if abs(abd[a(l, k)]) > 1.0e-15:
            if l != m:
                abd[a(l, k)], abd[a(m, k)] = abd[a(m, k)], abd[a(l, k)]
            t = -1.0 / abd[a(m, k)]
            abd[m:m + lm, k - 1] *= t
            ju = min(max(ju, ku + int(piv[k - 1])), n)
            mm = m
            for j in range(k + 1, ju + 1):
                l -= 1
                mm -= 1
                t = abd[a(l, j)]
                if l != mm:
                    abd[a(l, j)] = abd[a(mm, j)]
                    abd[a(mm, j)] = t
                abd[mm:mm + lm, j - 1] += t * abd[m:m + lm, k - 1]
        else:
            raise np.linalg.LinAlgError(f"singular band matrix at column {k}")
    piv[n - 1] = n
    return abd, piv


def band_solve(abd, piv, kl, ku, rhs):
    """solve_band_real (magic_torch/algebra.py:460-510, LINPACK dgbsl order) for the
    columns of rhs (n, ncol), real or complex."""
    x = np.array(rhs, dtype=rhs.dtype, copy=True)
    n = x.shape[0]
    m = kl + ku + 1
    if kl:
        for k in range(1, n):
            lm = min(kl, n - k)
            l = int(piv[k - 1])
            if l != k:
                x[[k - 1, l - 1]] = x[[l - 1, k - 1]]
            x[k:k + lm] += x[k - 1:k] * abd[m:m + lm, k - 1:k]
    for k in range(n, 0, -1):
        x[k - 1] = x[k - 1] / abd[m - 1, k - 1]
        lm = min(k, m) - 1
        la, lb = m - lm, k - lm
        if lm > 0:
            t = -x[k - 1:k]
            x[lb - 1:lb - 1 + lm] += t * abd[la - 1:la - 1 + lm, k - 1:k]
    return x


def _solve(dat, rhs, fac_row, fac_col=None, band=None):
    """Rows rhs (count, n) of one degree through the preconditioned matrix dat:
    np.linalg.solve, or the reference's banded LU (band = (kl, ku)) where it
    factorises (finite differences of order > 2, banded_solve_by_l,
    magic_torch/algebra.py:672-728)."""
    b = fac_row[None, :] * rhs
    if band is None:
        y = np.linalg.solve(dat, b.T).T
    else:
        abd, piv = band_factor(dat, *band)
        y = band_solve(abd, piv, band[0], band[1], b.T).T
    return y if fac_col is None else fac_col[None, :] * y


def _bw(fd_order, fd_order_bound):
    """Band width kl = ku of the S, Z, B and J matrices (update_s.py:97-104)."""
    return max(fd_order // 2, fd_order_bound)


def cnab2_weights(dt1, dt2, alpha=0.6):
    """wimp, wimp_lin, wexp of CNAB2 (magic_torch/time_scheme.py:56-73)."""
    return ([1.0], [alpha * dt1, (1.0 - alpha) * dt1],
            [(1.0 + 0.5 * dt1 / dt2) * dt1, -0.5 * dt1 * dt1 / dt2])


def s_matrix(l, mats, prof, wimp_lin0, opr, hdif_l, n_cheb):
    """Entropy LHS of degree l (magic_torch/update_s.py:67-134): rows 1..N-2 are
    rnorm (rMat - wimp opr hdif kappa (d2rMat + (beta + dLtemp0 + 2/r + dLkappa) drMat
    - l(l+1)/r^2 rMat)), rows 0 and N-1 the Dirichlet rows rnorm rMat, Chebyshev
    columns >= n_cheb zeroed in those rows, columns 0 and N-1 scaled by boundary_fac."""
    rMat, drMat, d2rMat, rnorm, bfac = mats
    N = rMat.shape[0]
    d1c = (prof["beta"] + prof["dLtemp0"] + 2.0 * prof["or1"] + prof["dLkappa"])[:, None]
    dL = float(l * (l + 1))
    dat = rnorm * (rMat - wimp_lin0 * opr * hdif_l * prof["kappa"][:, None] * (
        d2rMat + d1c * drMat - dL * prof["or2"][:, None] * rMat))
    dat[0, :] = rnorm * rMat[0, :]
    dat[N - 1, :] = rnorm * rMat[N - 1, :]
    if n_cheb < N:
        dat[0, n_cheb:] = 0.0
        dat[N - 1, n_cheb:] = 0.0
    dat[:, 0] *= bfac
    dat[:, N - 1] *= bfac
    return dat


def update_s(g, mats, prof, st, weights, opr, hdif, tops, bots, D1, D2, chebyshev, n_cheb,
             fd_order=2, fd_order_bound=2):
    """One updateS (magic_torch/update_s.py:213-271): CNAB2 right-hand side
    (time_scheme.py:82-96) with the boundary values in rows 0 and N-1, a solve per
    degree l (row-preconditioned LU), m = 0 coefficients made real, the DCT-I to
    grid values (Chebyshev only), then ds, d2s and the implicit term
    opr hdif kappa (d2s + (beta + dLtemp0 + 2/r + dLkappa) ds - l(l+1)/r^2 s).

    st: dict old, impl, expl0, expl1 ((lm_max, N) complex).  Returns s, ds, impl,
    old, expl1 after the update (expl0 is left for the next explicit stage)."""
    wimp, wimp_lin, wexp = weights
    N = st["old"].shape[1]
    rhs = wimp[0] * st["old"] + wimp_lin[1] * st["impl"] + wexp[0] * st["expl0"] \
        + wexp[1] * st["expl1"]
    rhs[:, 0] = tops
    rhs[:, N - 1] = bots
    x = np.empty_like(rhs)
    band = None if chebyshev or fd_order <= 2 else (_bw(fd_order, fd_order_bound),) * 2
    for l in range(g["l_max"] + 1):
        rows = np.nonzero(g["lm2l"] == l)[0]
        dat = s_matrix(l, mats, prof, wimp_lin[0], opr, hdif[l], n_cheb)
        fac = 1.0 / np.abs(dat).max(axis=1)
        x[rows] = _solve(fac[:, None] * dat, rhs[rows], fac, band=band)
    m0 = g["lm2m"] == 0
    x[m0] = x[m0].real
    if chebyshev:
        if n_cheb < N:
            x[:, n_cheb:] = 0.0
        x = x @ dct1_matrix(N).T
    ds, d2s = x @ D1.T, x @ D2.T
    d1c = prof["beta"] + prof["dLtemp0"] + 2.0 * prof["or1"] + prof["dLkappa"]
    dLh = (g["lm2l"] * (g["lm2l"] + 1.0))[:, None]
    impl = opr * hdif[g["lm2l"]][:, None] * prof["kappa"][None, :] * (
        d2s + d1c[None, :] * ds - dLh * prof["or2"][None, :] * x)
    return dict(s=x, ds=ds, impl=impl, old=x.copy(), expl1=st["expl0"].copy())


def z_matrix(l, mats, prof, wimp_lin0, hdif_l, n_cheb, ktopv, kbotv):
    """Toroidal-velocity LHS of degree l >= 1 (magic_torch/update_z.py:156-188):
    rnorm l(l+1)/r^2 (rMat - wimp hdif visc (d2rMat + (dLvisc - beta) drMat
    - (dLvisc beta + 2 dLvisc/r + l(l+1)/r^2 + dbeta + 2 beta/r) rMat)); boundary rows
    stress-free (k = 1: rnorm (drMat - (2/r + beta) rMat)) or no-slip (rnorm rMat)."""
    rMat, drMat, d2rMat, rnorm, bfac = mats
    N = rMat.shape[0]
    p = prof
    dL = float(l * (l + 1))
    c0 = (p["dLvisc"] * p["beta"] + 2.0 * p["dLvisc"] * p["or1"] + dL * p["or2"] + p["dbeta"]
          + 2.0 * p["beta"] * p["or1"])[:, None]
    dat = rnorm * dL * p["or2"][:, None] * (rMat - wimp_lin0 * hdif_l * p["visc"][:, None] * (
        d2rMat + (p["dLvisc"] - p["beta"])[:, None] * drMat - c0 * rMat))
    for row, k in ((0, ktopv), (N - 1, kbotv)):
        if k == 1:
            dat[row, :] = rnorm * (drMat[row, :] - (2.0 * p["or1"][row] + p["beta"][row]) * rMat[row, :])
        else:
            dat[row, :] = rnorm * rMat[row, :]
    if n_cheb < N:
        dat[0, n_cheb:] = 0.0
        dat[N - 1, n_cheb:] = 0.0
    dat[:, 0] *= bfac
    dat[:, N - 1] *= bfac
    return dat


def update_z(g, mats, prof, st, weights, hdif, D1, D2, chebyshev, n_cheb, ktopv, kbotv, fd_order,
             fd_order_bound=2):
    """One updateZ without inner-core rotation (magic_torch/update_z.py:333-505):
    CNAB2 right-hand side with zero boundary rows, per-l solves (l = 0: zero on the
    dense paths, the right-hand side itself on the banded finite-difference path,
    fd_order > 2), m = 0 real, DCT-I (Chebyshev), dz, d2z; old = l(l+1)/r^2 z and
    impl = hdif l(l+1)/r^2 visc (d2z + (dLvisc - beta) dz
    - (dLvisc beta + 2 dLvisc/r + dbeta + 2 beta/r + l(l+1)/r^2) z)."""
    wimp, wimp_lin, wexp = weights
    N = st["old"].shape[1]
    rhs = wimp[0] * st["old"] + wimp_lin[1] * st["impl"] + wexp[0] * st["expl0"] \
        + wexp[1] * st["expl1"]
    rhs[:, 0] = 0.0
    rhs[:, N - 1] = 0.0
    x = np.zeros_like(rhs)
    for l in range(g["l_max"] + 1):
        rows = np.nonzero(g["lm2l"] == l)[0]
        if l == 0:
            if not chebyshev and fd_order > 2:
                x[rows] = rhs[rows]
            continue
        dat = z_matrix(l, mats, prof, wimp_lin[0], hdif[l], n_cheb, ktopv, kbotv)
        fac = 1.0 / np.abs(dat).max(axis=1)
        band = None if chebyshev or fd_order <= 2 else (_bw(fd_order, fd_order_bound),) * 2
        x[rows] = _solve(fac[:, None] * dat, rhs[rows], fac, band=band)
    m0 = g["lm2m"] == 0
    x[m0] = x[m0].real
    if chebyshev:
        if n_cheb < N:
            x[:, n_cheb:] = 0.0
        x = x @ dct1_matrix(N).T
    dz, d2z = x @ D1.T, x @ D2.T
    p = prof
    dLh = (g["lm2l"] * (g["lm2l"] + 1.0))[:, None]
    z0 = (p["dLvisc"] * p["beta"] + 2.0 * p["dLvisc"] * p["or1"] + p["dbeta"]
          + 2.0 * p["beta"] * p["or1"])[None, :]
    or2 = p["or2"][None, :]
    impl = hdif[g["lm2l"]][:, None] * dLh * or2 * p["visc"][None, :] * (
        d2z + (p["dLvisc"] - p["beta"])[None, :] * dz - (z0 + dLh * or2) * x)
    return dict(x=x, dx=dz, impl=impl, old=dLh * or2 * x, expl1=st["expl0"].copy())


def b_matrices(l, mats, prof, wimp_lin0, opm, hdif_l, n_cheb):
    """Poloidal (b) and toroidal (j) magnetic LHS of degree l >= 1 with an
    insulating inner core (magic_torch/update_b.py:160-240): bulk rows
    rnorm l(l+1)/r^2 (rMat - wimp opm lambda hdif (d2rMat [+ dLlambda drMat for j]
    - l(l+1)/r^2 rMat)); b: rows rnorm (drMat + l/r rMat) at the top, rnorm (drMat
    - (l+1)/r rMat) at the bottom; j: Dirichlet rows."""
    rMat, drMat, d2rMat, rnorm, bfac = mats
    N = rMat.shape[0]
    p = prof
    dL = float(l * (l + 1))
    out = []
    for with_dl in (False, True):
        inner = d2rMat - dL * p["or2"][:, None] * rMat
        if with_dl:
            inner = inner + p["dLlambda"][:, None] * drMat
        dat = rnorm * dL * p["or2"][:, None] * (
            rMat - wimp_lin0 * opm * p["lambda_"][:, None] * hdif_l * inner)
        if with_dl:
            dat[0, :] = rnorm * rMat[0, :]
            dat[N - 1, :] = rnorm * rMat[N - 1, :]
        else:
            dat[0, :] = rnorm * (drMat[0, :] + l * p["or1"][0] * rMat[0, :])
            dat[N - 1, :] = rnorm * (drMat[N - 1, :] - (l + 1) * p["or1"][N - 1] * rMat[N - 1, :])
        if n_cheb < N:
            dat[0, n_cheb:] = 0.0
            dat[N - 1, n_cheb:] = 0.0
        dat[:, 0] *= bfac
        dat[:, N - 1] *= bfac
        out.append(dat)
    return out


def update_b(g, mats, prof, stb, stj, weights, opm, hdif, D1, D2, chebyshev, n_cheb, fd_order,
             fd_order_bound=2):
    """One updateB with an insulating inner core (magic_torch/update_b.py:530-635):
    both fields as update_z with their own matrices (degree 0 as there), old =
    l(l+1)/r^2 x and impl = opm lambda hdif l(l+1)/r^2 (d2x [+ dLlambda dx for j]
    - l(l+1)/r^2 x).  Returns the dicts of b and j (x, dx, d2x, impl, old, expl1)."""
    wimp, wimp_lin, wexp = weights
    N = stb["old"].shape[1]
    res = []
    for fi, st in enumerate((stb, stj)):
        rhs = wimp[0] * st["old"] + wimp_lin[1] * st["impl"] + wexp[0] * st["expl0"] \
            + wexp[1] * st["expl1"]
        rhs[:, 0] = 0.0
        rhs[:, N - 1] = 0.0
        x = np.zeros_like(rhs)
        for l in range(g["l_max"] + 1):
            rows = np.nonzero(g["lm2l"] == l)[0]
            if l == 0:
                if not chebyshev and fd_order > 2:
                    x[rows] = rhs[rows]
                continue
            dat = b_matrices(l, mats, prof, wimp_lin[0], opm, hdif[l], n_cheb)[fi]
            fac = 1.0 / np.abs(dat).max(axis=1)
            band = None if chebyshev or fd_order <= 2 else (_bw(fd_order, fd_order_bound),) * 2
            x[rows] = _solve(fac[:, None] * dat, rhs[rows], fac, band=band)
        m0 = g["lm2m"] == 0
        x[m0] = x[m0].real
        if chebyshev:
            if n_cheb < N:
                x[:, n_cheb:] = 0.0
            x = x @ dct1_matrix(N).T
        dx, d2x = x @ D1.T, x @ D2.T
        dLh = (g["lm2l"] * (g["lm2l"] + 1.0))[:, None]
        or2 = prof["or2"][None, :]
        inner = d2x - dLh * or2 * x
        if fi:
            inner = inner + prof["dLlambda"][None, :] * dx
        impl = opm * prof["lambda_"][None, :] * hdif[g["lm2l"]][:, None] * dLh * or2 * inner
        res.append(dict(x=x, dx=dx, d2x=d2x, impl=impl, old=dLh * or2 * x,
                        expl1=st["expl0"].copy()))
    return res


def _w_coefficients(prof, dL):
    """c3, c2, c1, c0 of the double-curl diffusion operator
    (magic_torch/update_w_doublecurl.py:137-190, 340-366)."""
    p = prof
    dLv, ddLv, b, db, ddb, or1, or2 = (p["dLvisc"], p["ddLvisc"], p["beta"], p["dbeta"],
                                       p["ddbeta"], p["or1"], p["or2"])
    c3 = 2.0 * (dLv - b)
    c2 = ddLv - 2.0 * db + dLv ** 2 + b ** 2 - 3.0 * dLv * b - 2.0 * or1 * (dLv + b) \
        - 2.0 * dL * or2
    c1 = (-ddb - db * (2.0 * dLv - b + 2.0 * or1) - ddLv * (b + 2.0 * or1)
          + b ** 2 * (dLv + 2.0 * or1) - b * (dLv ** 2 - 2.0 * or2)
          - 2.0 * dLv * or1 * (dLv - or1) + 2.0 * (2.0 * or1 + b - dLv) * dL * or2)
    c0 = dL * or2 * (2.0 * db + ddLv + dLv ** 2 - (2.0 / 3.0) * b ** 2 + dLv * b
                     + 2.0 * or1 * (2.0 * dLv - b - 3.0 * or1) + dL * or2)
    return c3, c2, c1, c0


def w_matrix(l, mats, prof, wimp_lin0, hdif_l, ktopv, kbotv):
    """Double-curl poloidal LHS of degree l >= 1 on finite-difference grid values
    (magic_torch/update_w_doublecurl.py:137-260): rows 2..N-3
    -l(l+1)/r^2/rho (d2 - beta d - l(l+1)/r^2) + wimp hdif visc l(l+1)/r^2/rho
    (d4 + c3 d3 + c2 d2 + c1 d + c0); rows 0, N-1: w = 0; rows 1, N-2: dw = 0
    (no-slip) or d2w - (2/r + beta) dw = 0 (stress-free) at the boundary."""
    rMat, drMat, d2rMat, d3rMat, d4rMat = mats
    N = rMat.shape[0]
    p = prof
    dL = float(l * (l + 1))
    b = slice(2, N - 2)
    c3, c2, c1, c0 = _w_coefficients(prof, dL)
    dat = np.zeros((N, N))
    old = (-dL * p["or2"] * p["orho1"])[b, None] * (
        d2rMat[b] - p["beta"][b, None] * drMat[b] - dL * p["or2"][b, None] * rMat[b])
    imp = (p["orho1"] * hdif_l * p["visc"] * dL * p["or2"])[b, None] * (
        d4rMat[b] + c3[b, None] * d3rMat[b] + c2[b, None] * d2rMat[b] + c1[b, None] * drMat[b]
        + c0[b, None] * rMat[b])
    dat[b] = old + wimp_lin0 * imp
    dat[0] = rMat[0]
    dat[N - 1] = rMat[N - 1]
    dat[1] = (d2rMat[0] - (2.0 * p["or1"][0] + p["beta"][0]) * drMat[0]) if ktopv == 1 else drMat[0]
    dat[N - 2] = ((d2rMat[N - 1] - (2.0 * p["or1"][N - 1] + p["beta"][N - 1]) * drMat[N - 1])
                  if kbotv == 1 else drMat[N - 1])
    return dat


def p0_matrix(mats, prof, r, fd_order):
    """l = 0 pressure matrix on finite-difference grid values
    (magic_torch/update_wp.py:80-140): rows 1.. dp/dr - beta p, last row the
    first-order backward difference (entries outside the band of width
    fd_order/2 dropped), row 0 the Dirichlet condition p = 0."""
    rMat, drMat = mats[0], mats[1]
    N = rMat.shape[0]
    dat = np.zeros((N, N))
    dat[1:] = drMat[1:] - prof["beta"][1:, None] * rMat[1:]
    delr = r[N - 1] - r[N - 2]
    dat[N - 1, N - 1] = 1.0 / delr - prof["beta"][N - 1]
    dat[N - 1, N - 2] = -1.0 / delr
    dat[N - 1, :N - 1 - fd_order // 2] = 0.0
    dat[0] = rMat[0]
    return dat


def update_w(g, mats, prof, st, weights, hdif, D1, D2, s_new, BuoFac, r, fd_order,
             ktopv, kbotv):
    """One double-curl updateW on finite differences (magic_torch/update_w_doublecurl.py:
    393-483): CNAB2 right-hand side plus wimp BuoFac l(l+1)/r^2 g s on rows 2..N-3,
    four boundary rows zero, degree 0 zero, per-l solves, m = 0 real; dw, ddw,
    dddw = D1 ddw, ddddw = D2 ddw; the l = 0 pressure from rho0 BuoFac g s00 +
    Re expl0; old and impl as get_w_old / get_w_impl."""
    # n_bands = max(fd_order + 3, 2 fd_order_bound + 3) (update_w_doublecurl.py:111-117);
    # banded LU where the reference factorises (fd_order > 2)
    wband = None if fd_order <= 2 else ((max(fd_order + 3, 2 * 2 + 3) - 1) // 2,) * 2
    wimp, wimp_lin, wexp = weights
    N = st["old"].shape[1]
    p = prof
    dLh = (g["lm2l"] * (g["lm2l"] + 1.0))[:, None]
    rhs = wimp[0] * st["old"] + wimp_lin[1] * st["impl"] + wexp[0] * st["expl0"] \
        + wexp[1] * st["expl1"]
    rhs[:, 2:N - 2] += wimp_lin[0] * BuoFac * dLh * (p["or2"] * p["rgrav"])[None, 2:N - 2] \
        * s_new[:, 2:N - 2]
    rhs[:, [0, 1, N - 2, N - 1]] = 0.0
    x = np.zeros_like(rhs)
    for l in range(1, g["l_max"] + 1):
        rows = np.nonzero(g["lm2l"] == l)[0]
        dat = w_matrix(l, mats, prof, wimp_lin[0], hdif[l], ktopv, kbotv)
        fr = 1.0 / np.abs(dat).max(axis=1)  # row, then column scaling as the reference
        dat = fr[:, None] * dat
        fc = 1.0 / np.abs(dat).max(axis=0)
        x[rows] = _solve(dat * fc[None, :], rhs[rows], fr, fc, band=wband)
    m0 = g["lm2m"] == 0
    x[m0] = x[m0].real
    dw, ddw = x @ D1.T, x @ D2.T
    dddw, ddddw = ddw @ D1.T, ddw @ D2.T
    p0_rhs = np.zeros(N)
    p0_rhs[1:] = p["rho0"][1:] * BuoFac * p["rgrav"][1:] * s_new[0, 1:].real + st["expl0"][0, 1:].real
    p0 = np.linalg.solve(p0_matrix(mats, prof, r, fd_order), p0_rhs)
    or2 = p["or2"][None, :]
    old = dLh * or2 * (-p["orho1"][None, :] * (ddw - p["beta"][None, :] * dw - dLh * or2 * x))
    old[:, [0, -1]] = 0.0
    c3, c2, c1, c0 = (np.broadcast_to(c, x.shape) for c in _w_coefficients(
        {k: v[None, :] if np.ndim(v) else v for k, v in prof.items()}, dLh))
    dif = -hdif[g["lm2l"]][:, None] * dLh * or2 * p["visc"][None, :] * p["orho1"][None, :] * (
        ddddw + c3 * dddw + c2 * ddw + c1 * dw + c0 * x)
    impl = dif + BuoFac * dLh * or2 * p["rgrav"][None, :] * s_new
    impl[:, [0, -1]] = 0.0
    return dict(x=x, dx=dw, d2x=ddw, impl=impl, old=old, expl1=st["expl0"].copy(), p0=p0)


def wp_matrix(l, mats, d3rMat, prof, wimp_lin0, hdif_l, n_cheb, ktopv, kbotv):
    """Coupled (w, p) LHS of degree l >= 1 in the standard poloidal form
    (magic_torch/update_wp.py:197-329), unknowns the Chebyshev coefficients of w
    (columns 0..N-1) and p (columns N..2N-1):
      w rows 1..N-2   rnorm l(l+1) or2 (rMat - wimp hdif visc (d2rMat
                      + (2 dLvisc - beta/3) drMat - (l(l+1) or2 + 4/3 (dLvisc beta
                      + (3 dLvisc + beta) or1 + dbeta)) rMat)) | rnorm wimp (drMat - beta rMat)
      p rows N+1..2N-2  rnorm l(l+1) or2 (-drMat - wimp hdif visc (-d3rMat
                      + (beta - dLvisc) d2rMat + (l(l+1) or2 + dbeta + dLvisc beta
                      + 2 (dLvisc + beta) or1) drMat - l(l+1) or2 (2 or1 + dLvisc
                      + 2/3 beta) rMat)) | -rnorm wimp l(l+1) or2 rMat
      rows 0, N-1     w = 0;  rows N, 2N-1  dw = 0 (no-slip) or d2w - (2 or1 + beta) dw = 0
                      (stress-free) at the top / bottom,
    Chebyshev columns >= n_cheb dropped in the four boundary rows, the first and
    last column of each block scaled by boundary_fac."""
    rMat, drMat, d2rMat, rnorm, bfac = mats
    N = rMat.shape[0]
    p = {k: np.asarray(v, dtype=np.float64)[:, None] for k, v in prof.items()
         if np.ndim(v) == 1}
    or1, or2, beta, dbeta, visc, dLv = (p[k] for k in ("or1", "or2", "beta", "dbeta", "visc",
                                                       "dLvisc"))
    dL = float(l * (l + 1))
    b = slice(1, N - 1)
    dat = np.zeros((2 * N, 2 * N))
    dat[b, :N] = rnorm * dL * or2[b] * (rMat[b] - wimp_lin0 * hdif_l * visc[b] * (
        d2rMat[b] + (2.0 * dLv[b] - beta[b] / 3.0) * drMat[b]
        - (dL * or2[b] + 4.0 / 3.0 * (dLv[b] * beta[b] + (3.0 * dLv[b] + beta[b]) * or1[b]
                                      + dbeta[b])) * rMat[b]))
    dat[b, N:] = rnorm * wimp_lin0 * (drMat[b] - beta[b] * rMat[b])
    dat[N + 1:2 * N - 1, :N] = rnorm * dL * or2[b] * (-drMat[b] - wimp_lin0 * hdif_l * visc[b] * (
        -d3rMat[b] + (beta[b] - dLv[b]) * d2rMat[b]
        + (dL * or2[b] + dbeta[b] + dLv[b] * beta[b] + 2.0 * (dLv[b] + beta[b]) * or1[b])
        * drMat[b]
        - dL * or2[b] * (2.0 * or1[b] + dLv[b] + 2.0 / 3.0 * beta[b]) * rMat[b]))
    dat[N + 1:2 * N - 1, N:] = -rnorm * wimp_lin0 * dL * or2[b] * rMat[b]
    dat[0, :N] = rnorm * rMat[0]
    dat[N - 1, :N] = rnorm * rMat[N - 1]
    o1, bt = prof["or1"], prof["beta"]
    dat[N, :N] = rnorm * ((d2rMat[0] - (2.0 * o1[0] + bt[0]) * drMat[0]) if ktopv == 1
                          else drMat[0])
    dat[2 * N - 1, :N] = rnorm * ((d2rMat[N - 1] - (2.0 * o1[N - 1] + bt[N - 1]) * drMat[N - 1])
                                  if kbotv == 1 else drMat[N - 1])
    if n_cheb < N:
        for row in (0, N - 1, N, 2 * N - 1):
            dat[row, n_cheb:N] = 0.0
            dat[row, N + n_cheb:] = 0.0
    for c in (0, N - 1, N, 2 * N - 1):
        dat[:, c] *= bfac
    return dat


def p0_matrix_cheb(mats, prof, n_cheb):
    """l = 0 pressure matrix on Chebyshev coefficients, Boussinesq row 0
    (magic_torch/update_wp.py:80-165): rows 1.. rnorm (drMat - beta rMat), row 0
    the Dirichlet row rnorm rMat[0] with columns >= n_cheb dropped, the first and
    last column scaled by boundary_fac."""
    rMat, drMat, _, rnorm, bfac = mats
    N = rMat.shape[0]
    dat = np.zeros((N, N))
    dat[1:] = rnorm * (drMat[1:] - prof["beta"][1:, None] * rMat[1:])
    dat[0] = rnorm * rMat[0]
    if n_cheb < N:
        dat[0, n_cheb:] = 0.0
    dat[:, 0] *= bfac
    dat[:, N - 1] *= bfac
    return dat


def update_wp(g, mats, d3rMat, prof, stw, stp, weights, hdif, D1, D2, D3, s_new, BuoFac,
              n_cheb, ktopv, kbotv):
    """One standard-form updateWP on Chebyshev levels (magic_torch/update_wp.py:
    387-531): CNAB2 right-hand sides of the w and p equations, plus
    wimp BuoFac rho0 rgrav s on the interior w rows, boundary rows zero; a coupled
    solve per degree l >= 1 (row, then column scaling, as the reference), m = 0
    made real; the l = 0 pressure from rho0 BuoFac rgrav Re s00 + Re expl0_w;
    Chebyshev truncation and the DCT-I to grid values; dw, ddw, dddw, dp; old and
    implicit terms of both equations (update_wp.py:470-531).

    stw, stp: dict old, impl, expl0, expl1 of the w and p equations."""
    wimp, wimp_lin, wexp = weights
    N = stw["old"].shape[1]
    pr = prof
    rhs_of = lambda st: (wimp[0] * st["old"] + wimp_lin[1] * st["impl"] + wexp[0] * st["expl0"]
                         + wexp[1] * st["expl1"])
    rw, rp = rhs_of(stw), rhs_of(stp)
    rhs = np.zeros((rw.shape[0], 2 * N), dtype=np.complex128)
    rhs[:, 1:N - 1] = rw[:, 1:N - 1] + wimp_lin[0] * BuoFac * (
        pr["rho0"] * pr["rgrav"])[None, 1:N - 1] * s_new[:, 1:N - 1]
    rhs[:, N + 1:2 * N - 1] = rp[:, 1:N - 1]
    sol = np.zeros_like(rhs)
    for l in range(1, g["l_max"] + 1):
        rows = np.nonzero(g["lm2l"] == l)[0]
        dat = wp_matrix(l, mats, d3rMat, prof, wimp_lin[0], hdif[l], n_cheb, ktopv, kbotv)
        fr = 1.0 / np.abs(dat).max(axis=1)
        dat = fr[:, None] * dat
        fc = 1.0 / np.abs(dat).max(axis=0)
        y = np.linalg.solve(dat * fc[None, :], (fr[None, :] * rhs[rows]).T).T
        sol[rows] = fc[None, :] * y
    m0 = g["lm2m"] == 0
    sol[m0] = sol[m0].real
    wc, pc = sol[:, :N].copy(), sol[:, N:].copy()
    lm0 = int(np.nonzero((g["lm2l"] == 0) & m0)[0][0])
    p0_rhs = np.zeros(N)
    p0_rhs[1:] = pr["rho0"][1:] * BuoFac * pr["rgrav"][1:] * s_new[lm0, 1:].real \
        + stw["expl0"][lm0, 1:].real
    pc[lm0] = np.linalg.solve(p0_matrix_cheb(mats, prof, n_cheb), p0_rhs)
    if n_cheb < N:
        wc[:, n_cheb:] = 0.0
        pc[:, n_cheb:] = 0.0
    C = dct1_matrix(N)
    w, p = wc @ C.T, pc @ C.T
    dw, ddw, dddw, dp = w @ D1.T, w @ D2.T, w @ D3.T, p @ D1.T
    dLh = (g["lm2l"] * (g["lm2l"] + 1.0))[:, None]
    r1 = lambda k: np.asarray(pr[k], dtype=np.float64)[None, :]
    or1, or2, beta, dbeta, visc, dLv = (r1(k) for k in ("or1", "or2", "beta", "dbeta", "visc",
                                                        "dLvisc"))
    hd = hdif[g["lm2l"]][:, None]
    dif = hd * dLh * or2 * visc * (
        ddw + (2.0 * dLv - beta / 3.0) * dw
        - (dLh * or2 + 4.0 / 3.0 * (dbeta + dLv * beta + (3.0 * dLv + beta) * or1)) * w)
    w_impl = -dp + beta * p + dif + BuoFac * r1("rho0") * r1("rgrav") * s_new
    p_impl = dLh * or2 * p + hd * visc * dLh * or2 * (
        -dddw + (beta - dLv) * ddw
        + (dLh * or2 + dLv * beta + dbeta + 2.0 * (dLv + beta) * or1) * dw
        - dLh * or2 * (2.0 * or1 + 2.0 / 3.0 * beta + dLv) * w)
    return dict(w=w, dw=dw, ddw=ddw, p=p, dp=dp, w_old=dLh * or2 * w, w_impl=w_impl,
                w_expl1=stw["expl0"].copy(), p_old=-dLh * or2 * dw, p_impl=p_impl,
                p_expl1=stp["expl0"].copy())
