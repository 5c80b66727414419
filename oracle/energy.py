"""CPU restatement (numpy, FP64) of the outer-core energy integrals and the
radial integration rules.  Test infrastructure only: the library never
imports this module.

Pinned against the reference's own outputs (tests/golden/energy_*.npz and
step_fd.npz, made by tests/golden/make_golden.py from magic_torch itself).
"""

from collections import namedtuple

import numpy as np

EKin = namedtuple("EKin", "e_p e_t e_p_as e_t_as e_p_es e_t_es e_p_eas e_t_eas")
EMagOC = namedtuple("EMagOC", "e_p e_t e_p_as e_t_as e_p_os e_p_as_os "
                              "e_p_es e_t_es e_p_eas e_t_eas e_p_e e_p_as_e")


def simps_weights(r):
    """magic_torch/integration.py:73-121 (non-uniform Simpson; even n_r: mean of
    two sweeps closed by trapezoids) applied to the unit vectors."""
    r = np.asarray(r, dtype=np.float64)
    N = r.size

    def simps(f):
        def sweep(start):
            acc = 0.0
            for n in range(start, N - 1, 2):
                h2, h1 = r[n + 1] - r[n], r[n] - r[n - 1]
                acc += (h1 + h2) / 6.0 * (f[n - 1] * (2.0 * h1 - h2) / h1
                                          + f[n] * (h1 + h2) * (h1 + h2) / (h1 * h2)
                                          + f[n + 1] * (2.0 * h2 - h1) / h2)
            return acc
        if N % 2 == 1:
            return -sweep(1)
        res = 0.5 * (r[1] - r[0]) * (f[1] + f[0]) + sweep(2)
        res += 0.5 * (r[N - 1] - r[N - 2]) * (f[N - 1] + f[N - 2]) + sweep(1)
        return -0.5 * res

    return np.array([simps(e) for e in np.eye(N)])


def cheb_weights(n_r, radratio):
    """magic_torch/integration.py:18-70: Clenshaw-Curtis through the DCT-I
    (cosine_transform.py:18-45), rnorm = sqrt(2/(N-1)), boundary_fac = 1/2."""
    N = n_r - 1
    r_cmb, r_icb = 1.0 / (1.0 - radratio), radratio / (1.0 - radratio)
    drx = 2.0 / (r_cmb - r_icb)
    k = np.arange(n_r)[:, None]
    j = np.arange(n_r)[None, :]
    C = 2.0 * np.cos(np.pi * j * k / N)
    C[:, 0] = 1.0
    C[:, N] = (-1.0) ** np.arange(n_r)
    C /= np.sqrt(2.0 * N)
    w = np.zeros(n_r)
    for e in range(n_r):
        a = C @ (np.eye(n_r)[e] / drx)
        a[0] *= 0.5
        a[-1] *= 0.5
        ci = np.zeros(n_r)
        ci[0] = 1.0
        for n in range(2, n_r, 2):
            n1 = n + 1
            ci[n] = -1.0 / (n1 * (n1 - 2))
        w[e] = 2.0 * np.sqrt(2.0 / N) * (a * ci).sum()
    return w


def _cc2real(c, m):
    """output.py:82-89."""
    return np.where(m[:, None] == 0, c.real ** 2, 2.0 * (c.real ** 2 + c.imag ** 2))


def _parts(e_pol, e_tor, lm2l, lm2m, rint, mag):
    m0 = lm2m == 0
    lpm_even = (lm2l + lm2m) % 2 == 0
    l_even = lm2l % 2 == 0
    es_p, es_t = (~lpm_even, lpm_even) if mag else (lpm_even, ~lpm_even)
    eas_p, eas_t = (m0 & ~l_even, m0 & l_even) if mag else (m0 & l_even, m0 & ~l_even)
    I = lambda e, mask: float(rint @ e[mask].sum(axis=0))
    return (I(e_pol, slice(None)), I(e_tor, slice(None)), I(e_pol, m0), I(e_tor, m0),
            I(e_pol, es_p), I(e_tor, es_t), I(e_pol, eas_p), I(e_tor, eas_t))


def e_kin_full(w, dw, z, lm2l, lm2m, or2, orho1, rint):
    """get_e_kin_full (output.py:101-140)."""
    dL = (lm2l * (lm2l + 1.0))[:, None]
    e_pol = 0.5 * orho1[None, :] * dL * (dL * or2[None, :] * _cc2real(w, lm2m)
                                         + _cc2real(dw, lm2m))
    e_tor = 0.5 * orho1[None, :] * dL * _cc2real(z, lm2m)
    return EKin(*_parts(e_pol, e_tor, lm2l, lm2m, rint, False))


def e_mag_oc_full(b, db, aj, lm2l, lm2m, or2, LFfac, r_cmb, rint):
    """get_e_mag_oc_full (output.py:143-190), no external field."""
    dL = (lm2l * (lm2l + 1.0))[:, None]
    fac = 0.5 * LFfac
    e_pol = fac * dL * (dL * or2[None, :] * _cc2real(b, lm2m) + _cc2real(db, lm2m))
    e_tor = fac * dL * _cc2real(aj, lm2m)
    p = _parts(e_pol, e_tor, lm2l, lm2m, rint, True)
    l = lm2l.astype(np.float64)
    cc = _cc2real(b[:, :1], lm2m)[:, 0]
    os_ = 0.5 * LFfac / r_cmb * l * l * (l + 1.0) * cc
    e_p_os, e_p_as_os = float(os_.sum()), float(os_[lm2m == 0].sum())
    return EMagOC(p[0], p[1], p[2], p[3], e_p_os, e_p_as_os, p[4], p[5], p[6], p[7], 0.0, 0.0)
