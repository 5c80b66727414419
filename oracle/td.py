"""CPU restatement (numpy, FP64) of the spectral explicit terms of one time
step: get_td assembly, finish_exp radial derivatives, radial derivative
operators and the DCT-I.  Test infrastructure only: the library never
imports this module.

Pinned against the reference's own outputs (tests/golden/td_*.npz, made by
tests/golden/make_golden.py from magic_torch itself).

Array layout as in the reference: spectral fields (lm_max, n_r) complex128,
m-major lm order (lm = lStart[m] + l - m).
"""

import numpy as np


def clm(l, m):
    """sqrt((l+m)(l-m)/((2l-1)(2l+1))) for l > 0, else 0
    (magic_torch/horizontal_data.py:91-100)."""
    l = np.asarray(l, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    out = np.zeros(np.broadcast(l, m).shape)
    mask = l > 0
    lm_, mm = np.broadcast_to(l, out.shape)[mask], np.broadcast_to(m, out.shape)[mask]
    out[mask] = np.sqrt((lm_ + mm) * (lm_ - mm) / ((2 * lm_ - 1) * (2 * lm_ + 1)))
    return out


def lm_arrays(lm2l, lm2m):
    """dPhi, dLh, dTheta2-4 A/S (magic_torch/horizontal_data.py:103-130)."""
    lf = lm2l.astype(np.float64)
    mf = lm2m.astype(np.float64)
    c_l, c_lp1 = clm(lf, mf), clm(lf + 1, mf)
    d = dict(dPhi=1j * mf, dLh=lf * (lf + 1))
    d["dTh1S"] = (lf + 1) * c_l
    d["dTh1A"] = lf * c_lp1
    d["dTh2S"] = (lf - 1) * c_l
    d["dTh2A"] = (lf + 2) * c_lp1
    d["dTh3S"] = (lf - 1) * (lf + 1) * c_l
    d["dTh3A"] = lf * (lf + 2) * c_lp1
    d["dTh4S"] = d["dTh1S"] * (lf - 1) * lf
    d["dTh4A"] = d["dTh1A"] * (lf + 1) * (lf + 2)
    return d


def neighbours(lm2l, lm2m, l_max):
    """l-1 and l+1 neighbours of each lm at the same m (magic_torch/blocking.py:19-52):
    S = lm - 1 (self, with a zero coefficient, at l = m); A = lm + 1 (masked at l = l_max)."""
    lm = np.arange(lm2l.size)
    S = np.where(lm2l > lm2m, lm - 1, lm)
    A = np.where(lm2l < l_max, lm + 1, 0)
    maskA = (lm2l < l_max).astype(np.float64)
    return S, A, maskA


def radial_apply(D, f):
    """out[..., j] = sum_k D[j, k] f[..., k] (magic_torch/radial_derivatives.py:29-68,
    both the dense and the banded forms)."""
    return f @ D.T


def dct1_matrix(n_r):
    """Self-inverse DCT-I as a matrix (magic_torch/cosine_transform.py:18-45):
    y[k] = (f[0] + (-1)^k f[N] + 2 sum_{j=1}^{N-1} f[j] cos(j k pi / N)) / sqrt(2N)."""
    N = n_r - 1
    k = np.arange(n_r)[:, None]
    j = np.arange(n_r)[None, :]
    C = 2.0 * np.cos(np.pi * j * k / N)
    C[:, 0] = 1.0
    C[:, N] = (-1.0) ** np.arange(n_r)
    return C / np.sqrt(2.0 * N)


def get_td(g, ins, D1):
    """All explicit terms of radial_loop step 4 (magic_torch/step_time.py:1139-1176):
    get_td.py:58-308 then finish_exp_pol (update_wp.py:371-385), finish_exp_entropy
    (update_s.py:191-210), finish_exp_comp (update_xi.py:183-202), finish_exp_mag
    (update_b.py:514-528).

    g: dict with lm2l, lm2m, l_max, r, or1, or2, or4, orho1, beta, CorFac, l_anel,
    l_double_curl.  ins: Advr, Advt, Advp, w, dw, ddw, z, dz (lm_max, n_r) complex,
    plus VSr, VSt / VXir, VXit / VxBr, VxBt, VxBp for the entropy / composition /
    induction terms (each group only when present).  Returns a dict of outputs.
    """
    h = lm_arrays(g["lm2l"], g["lm2m"])
    S, A, mA = neighbours(g["lm2l"], g["lm2m"], g["l_max"])
    col = lambda x: np.asarray(x, dtype=np.complex128)[:, None]
    row = lambda x: np.asarray(x, dtype=np.float64)[None, :]
    or1, or2, or4 = row(g["or1"]), row(g["or2"]), row(g["or4"])
    r2 = row(g["r"] * g["r"])
    orho1, beta = row(g["orho1"]).astype(np.complex128), row(g["beta"]).astype(np.complex128)
    dLh, dPhi = col(h["dLh"]), col(h["dPhi"])
    gA = lambda f: f[A, :] * mA[:, None]
    gS = lambda f: f[S, :]
    CF = g["CorFac"]
    w, dw, ddw, z, dz = (ins[k] for k in ("w", "dw", "ddw", "z", "dz"))
    out = {}

    def bnd0(x):
        x[:, 0] = 0.0
        x[:, -1] = 0.0
        return x

    if g["l_double_curl"]:
        # get_td.py:88-148
        dwdt = dLh * or4 * orho1 * ins["Advr"]
        dVxVh = -orho1 * r2 * dLh * ins["Advt"]
        zA, zS, dzA, dzS = gA(z), gS(z), gA(dz), gS(dz)
        cor = 2.0 * CF * or2 * orho1 * (
            dPhi * (-ddw + beta * dw + (beta * or1 + or2) * dLh * w)
            + col(h["dTh3A"]) * (dzA - beta * zA)
            + col(h["dTh3S"]) * (dzS - beta * zS)
            + or1 * (col(h["dTh4A"]) * zA - col(h["dTh4S"]) * zS))
        dwdt = dwdt + cor
        dwdt[0, :] = or2[0, :] * ins["Advr"][0, :]
        dwdt[0, :] += 2.0 * CF * or1[0, :] * h["dTh2A"][0] * z[A[0], :] * mA[0]
        bnd0(dwdt)
        bnd0(dVxVh)
        out["dwdt"] = dwdt + or2 * radial_apply(D1, dVxVh)
    else:
        # get_td.py:58-85
        dwdt = or2 * ins["Advr"]
        dwdt = dwdt + 2.0 * CF * or1 * (dPhi * dw + col(h["dTh2A"]) * gA(z)
                                        - col(h["dTh2S"]) * gS(z))
        out["dwdt"] = bnd0(dwdt)
        # get_td.py:184-213
        dpdt = -dLh * ins["Advt"]
        dpdt = dpdt + 2.0 * CF * or2 * (-dPhi * (dw + or1 * dLh * w)
                                        + col(h["dTh3A"]) * gA(z) + col(h["dTh3S"]) * gS(z))
        out["dpdt"] = bnd0(dpdt)
    # get_td.py:151-181
    dzdt = dLh * ins["Advp"]
    dzdt = dzdt + 2.0 * CF * or2 * (dPhi * z + col(h["dTh3A"]) * gA(dw)
                                    + or1 * col(h["dTh4A"]) * gA(w)
                                    + col(h["dTh3S"]) * gS(dw)
                                    - or1 * col(h["dTh4S"]) * gS(w))
    out["dzdt"] = bnd0(dzdt)
    # get_td.py:216-237 + update_s.py:191-210 (and the composition twin)
    for part, radial, name in (("VSt", "VSr", "dsdt"), ("VXit", "VXir", "dxidt")):
        if part not in ins:
            continue
        d = bnd0(dLh * ins[part])
        q = bnd0(ins[radial].copy())
        res = d - or2 * radial_apply(D1, q)
        if g["l_anel"]:
            res = orho1 * res
        out[name] = res
    # get_td.py:266-308 + update_b.py:514-528
    if "VxBp" not in ins:
        return out
    out["dbdt"] = bnd0(dLh * ins["VxBp"])
    dj = bnd0(dLh * or4 * ins["VxBr"])
    dVxBh = -dLh * ins["VxBt"] * r2
    dVxBh[0, 0] = 0.0
    dVxBh[0, -1] = 0.0
    out["djdt"] = dj + or2 * radial_apply(D1, dVxBh)
    return out
