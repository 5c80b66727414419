"""CPU port of the nonlinear stage with batched matrix products — CPU BASELINE ONLY.

TEST INFRASTRUCTURE / BASELINE ONLY (see ``oracle/__init__.py``): used by
``bench.py``'s CPU-baseline leg and checked against ``oracle.stage`` in the
tests.  It restates the reference's own CPU algorithm for speed rather than
for clarity: per-m Legendre matrices zero-padded to a common width and
contracted with one batched matmul per hemisphere and table
(``sht.py:78-175``, ``sht.py:298-405``), complex data viewed as real pairs.
Like the reference on the CPU, the batched products and phi FFTs run through
torch's CPU kernels (``torch.bmm``, ``torch.fft``) on all host threads;
get_nl and the Courant reduction use numpy broadcasting.
"""

import numpy as np
import torch

from . import grid as og
from . import nonlinear as onl


class FastGrid:
    def __init__(self, l_max, minc=1):
        g = og.Grid(l_max, minc)
        self.g = g
        for k in ("lm_max", "n_theta_max", "n_phi_max", "n_m_max", "NHS", "lm2l", "lm2m",
                  "dLh", "O_sin_theta_E2_grid", "gauss"):
            setattr(self, k, getattr(g, k))
        M, K, H = g.n_m_max, l_max + 1, g.NHS
        self.K = K
        idx = np.zeros((M, K), dtype=np.int64)
        valid = np.zeros((M, K), dtype=bool)
        for mc in range(M):
            n = g.lStop[mc] - g.lStart[mc] + 1
            idx[mc, :n] = np.arange(g.lStart[mc], g.lStop[mc] + 1)
            valid[mc, :n] = True
        self.idx, self.valid = idx, valid
        sgn = np.where(np.arange(K) % 2 == 0, 1.0, -1.0)
        P = np.where(valid[:, :, None], g.Plm[idx], 0.0)     # (M, K, H)
        dP = np.where(valid[:, :, None], g.dPlm[idx], 0.0)
        self.PN = np.ascontiguousarray(P.transpose(0, 2, 1))  # (M, H, K)
        self.PS = np.ascontiguousarray(self.PN * sgn)
        self.dPN = np.ascontiguousarray(dP.transpose(0, 2, 1))
        self.dPS = np.ascontiguousarray(-self.dPN * sgn)
        w = 2.0 * np.pi * g.gauss[:H]
        self.WN = np.ascontiguousarray(P * w)                  # (M, K, H)
        self.WS = np.ascontiguousarray(self.WN * sgn[None, :, None])
        self.dWN = np.ascontiguousarray(dP * w)
        self.dWS = np.ascontiguousarray(-self.dWN * sgn[None, :, None])
        self.m = (np.arange(M) * minc).astype(np.float64)

    # ---- helpers over (M, K, B) complex padded spectra
    def gather(self, X):
        return np.where(self.valid[:, :, None], X[self.idx], 0.0)

    @staticmethod
    def _mm(A, X):
        """real (M, a, b) @ complex (M, b, B) -> complex (M, a, B) via real pairs."""
        X = np.ascontiguousarray(X)
        Xr = torch.from_numpy(X.view(np.float64).reshape(X.shape[0], X.shape[1], -1))
        R = torch.bmm(torch.from_numpy(A), Xr).numpy()
        return R.reshape(R.shape[0], R.shape[1], -1, 2).view(np.complex128)[..., 0]

    def to_grid(self, FN, FS):
        """(M, H, B) north/south Fourier values -> (B, nt, np) grids."""
        M, H, B = FN.shape
        F = np.zeros((B, self.n_theta_max, self.n_phi_max // 2 + 1), dtype=np.complex128)
        F[:, 0::2, :M] = FN.transpose(2, 1, 0)
        F[:, 1::2, :M] = FS.transpose(2, 1, 0)
        return torch.fft.irfft(torch.from_numpy(F), n=self.n_phi_max, dim=2,
                               norm="forward").numpy()

    def fourier(self, x):
        F = torch.fft.rfft(torch.from_numpy(np.ascontiguousarray(x)), dim=2,
                           norm="forward")[:, :, :self.n_m_max].numpy()
        return (np.ascontiguousarray(F[:, 0::2].transpose(2, 1, 0)),
                np.ascontiguousarray(F[:, 1::2].transpose(2, 1, 0)))

    def scatter(self, Y):
        out = np.zeros((self.lm_max, Y.shape[2]), dtype=np.complex128)
        out[self.idx[self.valid]] = Y[self.valid]
        return out

    # ---- transforms
    def scal_to_spat(self, X):
        Xp = self.gather(X)
        return self.to_grid(self._mm(self.PN, Xp), self._mm(self.PS, Xp))

    def torpol_to_spat(self, Q, S, T):
        im = 1j * self.m[:, None, None]
        Qp, Sp, Tp = self.gather(Q), self.gather(S), self.gather(T)
        out = []
        br = self.to_grid(self._mm(self.PN, Qp), self._mm(self.PS, Qp))
        tN = self._mm(self.dPN, Sp) + im * self._mm(self.PN, Tp)
        tS = self._mm(self.dPS, Sp) + im * self._mm(self.PS, Tp)
        pN = im * self._mm(self.PN, Sp) - self._mm(self.dPN, Tp)
        pS = im * self._mm(self.PS, Sp) - self._mm(self.dPS, Tp)
        out = (br, self.to_grid(tN, tS), self.to_grid(pN, pS))
        return out

    def scal_to_SH(self, x):
        FN, FS = self.fourier(x)
        return self.scatter(self._mm(self.WN, FN) + self._mm(self.WS, FS))

    def spat_to_sphertor(self, vt, vp, want_t=True):
        ost2 = self.O_sin_theta_E2_grid
        tN, tS = self.fourier(vt * ost2[None, :, None])
        pN, pS = self.fourier(vp * ost2[None, :, None])
        mim = -1j * self.m[:, None, None]
        S = (self._mm(self.dWN, tN) + self._mm(self.dWS, tS)
             + mim * (self._mm(self.WN, pN) + self._mm(self.WS, pS)))
        inv = np.zeros(self.lm_max)
        inv[1:] = 1.0 / self.dLh[1:]
        S = self.scatter(S) * inv[:, None]
        if not want_t:
            return S, None
        T = (-(self._mm(self.dWN, pN) + self._mm(self.dWS, pS))
             + mim * (self._mm(self.WN, tN) + self._mm(self.WS, tS)))
        return S, self.scatter(T) * inv[:, None]


def nl_bouss_stage(fg, f, prof, LFfac, courfac, alffac, opm, l_mag=True, damp=True):
    """Same contract as ``oracle.stage.nl_bouss_stage`` (no composition)."""
    N = f["w"].shape[1]
    bulk = slice(1, N - 1)
    dLh = fg.dLh[:, None]
    or2 = np.asarray(prof["or2"])[None, :]
    sc = fg.scal_to_spat(f["s"])
    zeros = np.zeros_like(sc)
    if l_mag:
        br, bt, bp = fg.torpol_to_spat(dLh * f["b"], f["db"], f["aj"])
        cbr, cbt, cbp = fg.torpol_to_spat(dLh * f["aj"], f["dj"], or2 * dLh * f["b"] - f["ddb"])
    else:
        br = bt = bp = cbr = cbt = cbp = zeros
    vr, vt, vp = fg.torpol_to_spat(dLh * f["w"], f["dw"], f["z"])
    cvr, cvt, cvp = fg.torpol_to_spat(dLh * f["z"], f["dz"], or2 * dLh * f["w"] - f["ddw"])
    r = onl.get_nl(vr, vt, vp, cvr, cvt, cvp, sc, br, bt, bp, cbr, cbt, cbp, zeros,
                   prof["or2"], prof["or4"], fg.O_sin_theta_E2_grid, LFfac)
    Advr, Advt, Advp, VSr, VSt, VSp, VxBr, VxBt, VxBp = r[:9]
    out = {}

    def put(name, x):
        a = np.zeros((fg.lm_max, N), dtype=np.complex128)
        a[:, bulk] = x
        out[name] = a

    put("Advr", fg.scal_to_SH(Advr[bulk]))
    put("VSr", fg.scal_to_SH(VSr[bulk]))
    s_, t_ = fg.spat_to_sphertor(Advt[bulk], Advp[bulk])
    put("Advt", s_)
    put("Advp", t_)
    put("VSt", fg.spat_to_sphertor(VSt[bulk], VSp[bulk], want_t=False)[0])
    if l_mag:
        put("VxBr", fg.scal_to_SH(VxBr[bulk]))
        s_, t_ = fg.spat_to_sphertor(VxBt[bulk], VxBp[bulk])
        put("VxBt", s_)
        put("VxBp", t_)
    dtr, dth = onl.courant_check(vr, vt, vp, br if l_mag else None, bt, bp, courfac, alffac,
                                 prof["or2"], prof["or4"], prof["orho1"], prof["orho2"],
                                 fg.O_sin_theta_E2_grid, prof["delxr2"], prof["delxh2"], LFfac,
                                 opm, damp=damp)
    return out, dtr, dth
