"""CPU oracle: grid sizes, Gauss-Legendre nodes, lm maps, Legendre tables.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Plain numpy, FP64.

Restates:
* ``params.py:12-24``          smallest 2^i 3^j 5^k >= n (phi-grid size)
* ``params.py:57-76``          derived grid sizes
* ``horizontal_data.py:16-50`` Gauss-Legendre nodes/weights (Newton on P_n)
* ``horizontal_data.py:59-84`` interleaved N/S theta order and grid arrays
* ``blocking.py:19-52``        m-major (standard) lm ordering
* ``plms.py:21-155``           fully normalised P_l^m and sin(theta) dP/dtheta
* ``plms.py:158-209``          tables over the northern Gauss points, lStart/lStop
* ``horizontal_data.py:96-124`` dLh = l(l+1), dPhi = i m
"""

import math

import numpy as np


def prime_decomposition(n):
    """Smallest value 2^i 3^j 5^k >= n, i<13, j<7, k<7 (``params.py:12-24``)."""
    best, dist_min = n, None
    for i in range(13):
        for j in range(7):
            for k in range(7):
                val = 2 ** i * 3 ** j * 5 ** k
                d = val - n
                if d >= 0 and (dist_min is None or d < dist_min):
                    dist_min, best = d, val
    return best


def grid_sizes(l_max, minc=1):
    """Grid sizes derived from (l_max, minc) exactly as ``params.py:57-76``.

    Returns a dict with n_phi_tot, n_phi_max (points per sector), n_theta_max,
    n_m_max, lm_max.
    """
    nalias = 20
    n_phi_tot = prime_decomposition(2 * ((30 * l_max) // nalias))
    m_max = l_max
    return dict(
        l_max=l_max,
        minc=minc,
        n_phi_tot=n_phi_tot,
        n_phi_max=n_phi_tot // minc,
        n_theta_max=n_phi_tot // 2,
        n_m_max=m_max // minc + 1,
        lm_max=sum(l_max - m + 1 for m in range(0, m_max + 1, minc)),
    )


def gauleg(n):
    """Gauss-Legendre colatitudes and weights on [-1, 1] (``horizontal_data.py:16-50``).

    Newton iteration on P_n from the asymptotic guess cos(pi (i-1/4)/(n+1/2)),
    stopping when the update is below 10 * eps.  Vectorised over the roots:
    each root keeps iterating only while its own update exceeds eps.
    Returns (theta_ord, gauss), theta_ord ascending (north pole first).
    """
    eps = 10.0 * np.finfo(np.float64).eps
    half = (n + 1) // 2
    i = np.arange(1, half + 1, dtype=np.float64)
    z = np.cos(math.pi * (i - 0.25) / (n + 0.5))
    z1 = z + 10.0 * eps
    pp = np.zeros_like(z)
    active = np.abs(z - z1) > eps
    while active.any():
        za = z[active]
        p1 = np.ones_like(za)
        p2 = np.zeros_like(za)
        for j in range(1, n + 1):
            p3 = p2
            p2 = p1
            p1 = ((2 * j - 1) * za * p2 - (j - 1) * p3) / j
        ppa = n * (za * p1 - p2) / (za * za - 1.0)
        pp[active] = ppa
        z1[active] = za
        z[active] = za - p1 / ppa
        active = np.abs(z - z1) > eps
    theta = np.zeros(n)
    gauss = np.zeros(n)
    idx = np.arange(half)
    theta[idx] = np.arccos(z)
    theta[n - 1 - idx] = np.arccos(-z)
    w = 2.0 / ((1.0 - z * z) * pp * pp)
    gauss[idx] = w
    gauss[n - 1 - idx] = w
    return theta, gauss


def lm_maps(l_max, minc=1):
    """m-major lm ordering (``blocking.py:19-52``; lStart/lStop ``plms.py:192-209``).

    Returns (lm2l, lm2m, lStart, lStop) with lStart[mc] the first lm of order
    m = mc*minc and lStop[mc] its last (l = l_max).
    """
    l_list, m_list, l_start, l_stop = [], [], [], []
    pos = 0
    for m in range(0, l_max + 1, minc):
        l_start.append(pos)
        for l in range(m, l_max + 1):
            l_list.append(l)
            m_list.append(m)
        pos += l_max - m + 1
        l_stop.append(pos - 1)
    return (np.array(l_list, dtype=np.int64), np.array(m_list, dtype=np.int64),
            np.array(l_start, dtype=np.int64), np.array(l_stop, dtype=np.int64))


def plm_tables(theta, l_max, minc=1):
    """P_l^m(cos theta) and sin(theta) dP_l^m/dtheta at the given colatitudes.

    Fully normalised with the 1/sqrt(4 pi) factor, no Condon-Shortley phase
    (``plms.py:21-155``, norm=2).  Vectorised over theta.  Returns two arrays of
    shape (lm_max, len(theta)) in m-major lm order.

    Recurrences (per order m):
      P_m^m      = sqrt(prod_{j=3,5..2m+1} j/(j-1)) sin^m(theta) / sqrt(4 pi)
      P_l^m      = cos(theta) a_lm P_{l-1}^m - b_lm P_{l-2}^m
                   a_lm = sqrt((2l-1)(2l+1)/((l-m)(l+m)))
                   b_lm = sqrt((2l+1)(l+m-1)(l-m-1)/((2l-3)(l-m)(l+m)))
      sin dP_l^m = l c_{l+1} P_{l+1}^m - (l+1) c_l P_{l-1}^m,
                   c_l = sqrt((l+m)(l-m)/((2l-1)(2l+1))),
    with P_{l_max+1}^m from one extra recurrence step.
    """
    theta = np.asarray(theta, dtype=np.float64)
    osq4pi = 1.0 / math.sqrt(4.0 * math.pi)
    cos_t = np.cos(theta)
    sin_t = np.sin(theta)
    ms = list(range(0, l_max + 1, minc))
    lm_max = sum(l_max - m + 1 for m in ms)
    P = np.zeros((lm_max, theta.size))
    dP = np.zeros((lm_max, theta.size))
    pos = 0
    for m in ms:
        fac = 1.0
        for j in range(3, 2 * m + 2, 2):
            fac = fac * j / (j - 1)
        pmm = math.sqrt(fac)
        plm = np.where(sin_t != 0.0, pmm * sin_t ** m, pmm if m == 0 else 0.0)
        n = l_max - m + 1
        col = np.zeros((n + 1, theta.size))  # P_m..P_{l_max+1}
        col[0] = plm
        plm1 = np.zeros_like(plm)
        for k, l in enumerate(range(m + 1, l_max + 2), start=1):
            plm2 = plm1
            plm1 = plm
            if (l - m) * (l + m) > 0:
                a = math.sqrt(float((2 * l - 1) * (2 * l + 1)) / float((l - m) * (l + m)))
                b = math.sqrt(float((2 * l + 1) * (l + m - 1) * (l - m - 1))
                              / float((2 * l - 3) * (l - m) * (l + m)))
                plm = cos_t * a * plm1 - b * plm2
            else:
                plm = np.zeros_like(plm1)
            col[k] = plm
        col *= osq4pi
        P[pos:pos + n] = col[:n]
        for k in range(n):
            l = m + k
            up = l * math.sqrt(float((l + m + 1) * (l - m + 1))
                               / float((2 * l + 1) * (2 * l + 3))) * col[k + 1]
            if k == 0:
                dP[pos + k] = up
            else:
                dn = (l + 1) * math.sqrt(float((l + m) * (l - m))
                                         / float((2 * l - 1) * (2 * l + 1))) * col[k - 1]
                dP[pos + k] = up - dn
        pos += n
    return P, dP


class Grid:
    """All horizontal tables for one (l_max, minc) resolution, FP64 on the CPU.

    Attributes mirror the reference's module globals: ``theta_ord``, ``gauss``
    (geographic order), ``Plm``/``dPlm``/``wPlm``/``wdPlm`` of shape
    (lm_max, NHS) over the northern points (``plms.py:158-186``), the
    interleaved-order arrays ``grid_idx``, ``O_sin_theta_E2_grid``,
    ``cosn_theta_E2_grid``, ``gauss_grid`` (``horizontal_data.py:59-84``), and
    ``dLh`` (``horizontal_data.py:110``).
    """

    def __init__(self, l_max, minc=1):
        s = grid_sizes(l_max, minc)
        self.__dict__.update(s)
        if self.n_theta_max % 2:
            raise ValueError("n_theta_max must be even")
        self.NHS = self.n_theta_max // 2
        self.theta_ord, self.gauss = gauleg(self.n_theta_max)
        self.lm2l, self.lm2m, self.lStart, self.lStop = lm_maps(l_max, minc)
        th_n = self.theta_ord[:self.NHS]
        self.Plm, self.dPlm = plm_tables(th_n, l_max, minc)
        w = 2.0 * math.pi * self.gauss[:self.NHS]
        self.wPlm = self.Plm * w[None, :]
        self.wdPlm = self.dPlm * w[None, :]
        # (l - m) even -> +1 (equatorially symmetric P), odd -> -1
        self.parity = np.where((self.lm2l - self.lm2m) % 2 == 0, 1.0, -1.0)
        gi = np.zeros(self.n_theta_max, dtype=np.int64)
        gi[0::2] = np.arange(self.NHS)
        gi[1::2] = np.arange(self.n_theta_max - 1, self.NHS - 1, -1)
        self.grid_idx = gi
        th = self.theta_ord[gi]
        self.theta_grid = th
        sin_g = np.sin(th)
        self.O_sin_theta_E2_grid = 1.0 / sin_g ** 2
        self.cosn_theta_E2_grid = np.cos(th) * self.O_sin_theta_E2_grid
        self.gauss_grid = self.gauss[gi]
        lf = self.lm2l.astype(np.float64)
        self.dLh = lf * (lf + 1.0)
        self.dPhi = 1j * self.lm2m.astype(np.float64)
