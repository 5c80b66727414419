"""Reference-signature transforms (drop-in for ``magic_torch.sht``).

Same names, argument meaning, shapes and dtypes as ``magic_torch/sht.py``;
``lcut`` is accepted and ignored there and here (always l_max).  All work runs
in ``libmagic_b200.so`` on the configured CUDA device (``magic_b200.config``).
"""

import torch

from .config import default_plan


def scal_to_spat(Slm, lcut=None):
    """magic_torch/sht.py:298-348"""
    return default_plan().scal_to_spat(Slm)


def scal_to_SH(sc, lcut=None):
    """magic_torch/sht.py:351-405"""
    return default_plan().scal_to_SH(sc)


def spat_to_SH(sc, lcut=None):
    """magic_torch/sht.py:570-572"""
    return default_plan().scal_to_SH(sc)


def torpol_to_spat(Qlm, Slm, Tlm, lcut=None):
    """magic_torch/sht.py:408-497"""
    return default_plan().torpol_to_spat(Qlm, Slm, Tlm)


def spat_to_sphertor(vt, vp, lcut=None):
    """magic_torch/sht.py:575-667"""
    return default_plan().spat_to_sphertor(vt, vp)


def scal_to_grad_spat(Slm, lcut=None):
    """magic_torch/sht.py:500-567"""
    return default_plan().scal_to_grad_spat(Slm)


def pol_to_grad_spat(Slm, lcut=None):
    """magic_torch/sht.py:706-722 (l(l+1) applied on load)"""
    return default_plan().pol_to_grad_spat(Slm)


def sphtor_to_spat(Slm, Tlm, lcut=None):
    """magic_torch/sht.py:670-684"""
    _, vt, vp = default_plan().torpol_to_spat(torch.zeros_like(Slm), Slm, Tlm)
    return vt, vp


def pol_to_curlr_spat(Qlm, lcut=None):
    """magic_torch/sht.py:687-703"""
    p = default_plan()
    d = p.dLh if Qlm.dim() == 1 else p.dLh.unsqueeze(1)
    return p.scal_to_spat(d * Qlm)


def torpol_to_dphspat(dWlm, Zlm, lcut=None):
    """magic_torch/sht.py:725-743"""
    p = default_plan()
    vt, vp = sphtor_to_spat(p.dPhi * dWlm, p.dPhi * Zlm)
    o = p.O_sin_theta_E2_grid.unsqueeze(1)
    return vt * o, vp * o


def torpol_to_curl_spat(or2, Blm, ddBlm, Jlm, dJlm, lcut=None):
    """magic_torch/sht.py:746-770"""
    p = default_plan()
    if Blm.dim() == 2:
        d = p.dLh.unsqueeze(1)
        o = torch.as_tensor(or2, dtype=torch.float64, device=p.device).unsqueeze(0)
        Q = d * Jlm
        T = o * d * Blm - ddBlm
    else:
        Q = p.dLh * Jlm
        T = float(or2) * p.dLh * Blm - ddBlm
    return p.torpol_to_spat(Q, dJlm, T)


def spat_to_qst(f, g, h, lcut=None):
    """magic_torch/sht.py:773-789"""
    p = default_plan()
    q = p.scal_to_SH(f)
    s, t = p.spat_to_sphertor(g, h)
    return q, s, t
