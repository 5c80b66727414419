"""CPU oracle: spherical-harmonic transforms (reference ``sht.py``).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Plain numpy, FP64.

Conventions reproduced (``sht.py:1-12``, ``sht.py:298-789``):
* spectral arrays are (lm_max,) or (lm_max, B) complex, m-major lm order;
* grid arrays are (n_theta, n_phi) or (B, n_theta, n_phi) real, theta rows in
  interleaved order [N0, S0, N1, S1, ...];
* synthesis is ``irfft(.., norm="forward")`` (unscaled), analysis
  ``rfft(.., norm="forward")`` (scaled by 1/n_phi); the FFT index is m/minc;
* the southern value of P_l^m is (-1)^(l-m) times the northern one and of
  sin(theta) dP/dtheta it is -(-1)^(l-m) times.

The vector transforms are written in the S/T form rather than the reference's
G = S - iT, C = S + iT stacks; the two are algebraically identical
(``sht.py:432-463`` and ``sht.py:626-661``):
    v_theta = sum_l [ dP S + i m P T ],     v_phi = sum_l [ i m P S - dP T ]
    S_lm    = sum_theta [ wdP V_theta - i m wP V_phi ] / (l(l+1))
    T_lm    = sum_theta [ -wdP V_phi - i m wP V_theta ] / (l(l+1))
with V = rfft(v) / sin^2(theta).
"""

import numpy as np


def _as_batched_spec(x):
    x = np.asarray(x)
    return (x[:, None], False) if x.ndim == 1 else (x, True)


def _as_batched_grid(x):
    x = np.asarray(x, dtype=np.float64)
    return (x[None], False) if x.ndim == 2 else (x, True)


def _hemisphere_tables(g, ls, le, table):
    """Northern and southern copies of one m-block of P (``table='P'``) or dP."""
    T = (g.Plm if table == "P" else g.dPlm)[ls:le + 1]
    par = g.parity[ls:le + 1][:, None]
    return T, (par * T if table == "P" else -par * T)


def _synth(g, terms, B):
    """Sum of Legendre syntheses into an (n_theta, n_phi//2+1, B) spectrum.

    ``terms`` is a list of (table, coef, X) with X (lm_max, B) complex and
    coef a function m -> complex scalar multiplying that table's sum.
    """
    F = np.zeros((g.n_theta_max, g.n_phi_max // 2 + 1, B), dtype=np.complex128)
    for mc in range(g.n_m_max):
        m = mc * g.minc
        ls, le = g.lStart[mc], g.lStop[mc]
        accN = np.zeros((g.NHS, B), dtype=np.complex128)
        accS = np.zeros((g.NHS, B), dtype=np.complex128)
        for table, coef, X in terms:
            TN, TS = _hemisphere_tables(g, ls, le, table)
            c = coef(m)
            Xm = X[ls:le + 1]
            accN += c * (TN.T @ Xm)
            accS += c * (TS.T @ Xm)
        F[0::2, mc] = accN
        F[1::2, mc] = accS
    return F


def _to_grid(g, F, batched):
    sc = np.fft.irfft(F, n=g.n_phi_max, axis=1, norm="forward")  # (nt, np, B)
    sc = np.transpose(sc, (2, 0, 1))
    return sc if batched else sc[0]


def _fourier(g, grid):
    """rfft over phi, norm='forward', kept modes m/minc < n_m_max: (B, nt, M)."""
    return np.fft.rfft(grid, axis=2, norm="forward")[:, :, :g.n_m_max]


def _analyse(g, terms, B):
    """Legendre analysis: sum_theta over both hemispheres of weighted tables.

    ``terms`` is a list of (table, coef, F) with F (B, n_theta, n_m) complex
    Fourier coefficients (interleaved theta rows) and table 'wP' or 'wdP'.
    Returns (lm_max, B) complex.
    """
    out = np.zeros((g.lm_max, B), dtype=np.complex128)
    par_all = g.parity
    for mc in range(g.n_m_max):
        m = mc * g.minc
        ls, le = g.lStart[mc], g.lStop[mc]
        par = par_all[ls:le + 1][:, None]
        acc = np.zeros((le - ls + 1, B), dtype=np.complex128)
        for table, coef, F in terms:
            W = (g.wPlm if table == "wP" else g.wdPlm)[ls:le + 1]
            WS = par * W if table == "wP" else -par * W
            FN = F[:, 0::2, mc].T  # (NHS, B)
            FS = F[:, 1::2, mc].T
            acc += coef(m) * (W @ FN + WS @ FS)
        out[ls:le + 1] = acc
    return out


def scal_to_spat(g, Slm):
    """Scalar synthesis (``sht.py:298-348``)."""
    X, batched = _as_batched_spec(Slm)
    F = _synth(g, [("P", lambda m: 1.0, X)], X.shape[1])
    return _to_grid(g, F, batched)


def scal_to_SH(g, sc):
    """Scalar analysis (``sht.py:351-405``)."""
    x, batched = _as_batched_grid(sc)
    F = _fourier(g, x)
    out = _analyse(g, [("wP", lambda m: 1.0, F)], x.shape[0])
    return out if batched else out[:, 0]


def torpol_to_spat(g, Qlm, Slm, Tlm):
    """Q/S/T synthesis to (b_r, b_theta, b_phi) (``sht.py:408-497``).

    The l=0 entries of S and T are ignored (``sht.py:434-435``).
    """
    Q, batched = _as_batched_spec(Qlm)
    S = _as_batched_spec(Slm)[0].astype(np.complex128).copy()
    T = _as_batched_spec(Tlm)[0].astype(np.complex128).copy()
    S[0] = 0.0
    T[0] = 0.0
    B = Q.shape[1]
    one = lambda m: 1.0
    im = lambda m: 1j * m
    Fr = _synth(g, [("P", one, Q)], B)
    Ft = _synth(g, [("dP", one, S), ("P", im, T)], B)
    Fp = _synth(g, [("P", im, S), ("dP", lambda m: -1.0, T)], B)
    return tuple(_to_grid(g, F, batched) for F in (Fr, Ft, Fp))


def scal_to_grad_spat(g, Slm):
    """(d/dtheta, 1/sin d/dphi) synthesis, sin-weighted (``sht.py:500-567``)."""
    X, batched = _as_batched_spec(Slm)
    B = X.shape[1]
    Ft = _synth(g, [("dP", lambda m: 1.0, X)], B)
    Fp = _synth(g, [("P", lambda m: 1j * m, X)], B)
    return _to_grid(g, Ft, batched), _to_grid(g, Fp, batched)


def spat_to_sphertor(g, vt, vp):
    """(v_theta, v_phi) analysis to (S, T), divided by l(l+1) (``sht.py:575-667``)."""
    xt, batched = _as_batched_grid(vt)
    xp, _ = _as_batched_grid(vp)
    ost2 = g.O_sin_theta_E2_grid[None, :, None]
    Ft = _fourier(g, xt) * ost2
    Fp = _fourier(g, xp) * ost2
    B = xt.shape[0]
    one = lambda m: 1.0
    mim = lambda m: -1j * m
    S = _analyse(g, [("wdP", one, Ft), ("wP", mim, Fp)], B)
    T = _analyse(g, [("wdP", lambda m: -1.0, Fp), ("wP", mim, Ft)], B)
    inv = np.zeros(g.lm_max)
    inv[1:] = 1.0 / g.dLh[1:]
    S *= inv[:, None]
    T *= inv[:, None]
    if not batched:
        return S[:, 0], T[:, 0]
    return S, T


def sphtor_to_spat(g, Slm, Tlm):
    """(S, T) to (v_theta, v_phi) (``sht.py:670-684``)."""
    _, vt, vp = torpol_to_spat(g, np.zeros_like(np.asarray(Slm)), Slm, Tlm)
    return vt, vp


def pol_to_curlr_spat(g, Qlm):
    """scal_to_spat(l(l+1) Q) (``sht.py:687-703``)."""
    Q = np.asarray(Qlm)
    d = g.dLh if Q.ndim == 1 else g.dLh[:, None]
    return scal_to_spat(g, d * Q)


def pol_to_grad_spat(g, Slm):
    """scal_to_grad_spat(l(l+1) S) (``sht.py:706-722``)."""
    S = np.asarray(Slm)
    d = g.dLh if S.ndim == 1 else g.dLh[:, None]
    return scal_to_grad_spat(g, d * S)


def torpol_to_dphspat(g, dWlm, Zlm):
    """phi-derivative fields, scaled by 1/sin^2 (``sht.py:725-743``)."""
    dW = np.asarray(dWlm)
    Z = np.asarray(Zlm)
    dphi = g.dPhi if dW.ndim == 1 else g.dPhi[:, None]
    vt, vp = sphtor_to_spat(g, dphi * dW, dphi * Z)
    ost2 = g.O_sin_theta_E2_grid
    ost2 = ost2[:, None] if vt.ndim == 2 else ost2[None, :, None]
    return vt * ost2, vp * ost2


def torpol_to_curl_spat(g, or2, Blm, ddBlm, Jlm, dJlm):
    """Curl of a toroidal/poloidal field (``sht.py:746-770``)."""
    B_ = np.asarray(Blm)
    if B_.ndim == 2:
        d = g.dLh[:, None]
        o = np.asarray(or2, dtype=np.float64)[None, :]
    else:
        d = g.dLh
        o = float(or2)
    Q = d * np.asarray(Jlm)
    T = o * d * B_ - np.asarray(ddBlm)
    return torpol_to_spat(g, Q, np.asarray(dJlm), T)


def spat_to_qst(g, f, gg, h):
    """(scal_to_SH(f), spat_to_sphertor(g, h)) (``sht.py:773-789``)."""
    q = scal_to_SH(g, f)
    s, t = spat_to_sphertor(g, gg, h)
    return q, s, t
