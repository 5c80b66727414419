"""Kinetic and magnetic energies of the outer core on the GPU (FP64).

The reference's get_e_kin_full and get_e_mag_oc_full
(magic_torch/output.py:101-190) through mt_energy: the spectral densities
are summed over lm under the reference's masks and integrated over r with
its radial rule (Simpson on the finite-difference grid, Clenshaw-Curtis on
Chebyshev points; RadialScheme.rint holds the rule as weights).  The results
are read back to the host (one small copy), as the reference's ``.item()``
calls do.
"""

import ctypes as C
from collections import namedtuple

import numpy as np
import torch

from . import _lib
from ._lib import check

EKin = namedtuple("EKin", "e_p e_t e_p_as e_t_as e_p_es e_t_es e_p_eas e_t_eas")
EMagOC = namedtuple("EMagOC", "e_p e_t e_p_as e_t_as e_p_os e_p_as_os "
                              "e_p_es e_t_es e_p_eas e_t_eas e_p_e e_p_as_e")


class EnergyIntegrals:
    """Energy integrals for one plan and radial grid.

    r, or2, orho1, rint: radial profiles (n_r); LFfac: the Lorentz-force factor
    1 / (Ek Pm) that scales the magnetic energy."""

    def __init__(self, plan, r, or2, orho1, rint, LFfac=1.0):
        self.plan = plan
        dev = plan.device
        t = lambda x: torch.as_tensor(np.asarray(x, dtype=np.float64), device=dev).contiguous()
        self.n_r = len(r)
        self.r_cmb = float(np.asarray(r, dtype=np.float64)[0])
        self.LFfac = float(LFfac)
        self.or2, self.rint = t(or2), t(rint)
        self.cr_kin = t(0.5 * np.asarray(orho1, dtype=np.float64))
        self.cr_mag = t(np.full(self.n_r, 0.5 * self.LFfac))
        nbytes = _lib.lib().mt_energy_workspace(plan._h)
        self.work = torch.empty(nbytes, dtype=torch.uint8, device=dev)

    def _run(self, pol, dpol, tor, cr, magnetic):
        for a in (pol, dpol, tor):
            if a.dim() != 2 or a.shape != (self.plan.lm_max, self.n_r) or \
                    a.dtype != torch.complex128 or a.stride(1) != 1:
                raise ValueError("fields must be (lm_max, n_r) complex128 with unit radial stride")
        if not (pol.stride(0) == dpol.stride(0) == tor.stride(0)):
            raise ValueError("fields must share their row stride")
        out = torch.empty(10, dtype=torch.float64, device=self.plan.device)
        e = _lib.EnergyArgs(pol.data_ptr(), dpol.data_ptr(), tor.data_ptr(), pol.stride(0),
                            self.or2.data_ptr(), cr.data_ptr(), self.rint.data_ptr(),
                            int(magnetic))
        st = C.c_void_p(torch.cuda.current_stream(self.plan.device).cuda_stream)
        check(_lib.lib().mt_energy(self.plan._h, self.n_r, C.byref(e), out.data_ptr(),
                                   self.work.data_ptr(), self.work.numel(), st))
        return out.cpu().tolist()

    def kin(self, w, dw, z):
        """get_e_kin_full(w, dw, z) (output.py:101-140)."""
        v = self._run(w, dw, z, self.cr_kin, False)
        return EKin(v[0], v[4], v[1], v[5], v[2], v[6], v[3], v[7])

    def mag(self, b, db, aj):
        """get_e_mag_oc_full(b, db, aj) (output.py:143-190); no external field."""
        v = self._run(b, db, aj, self.cr_mag, True)
        fos = 0.5 * self.LFfac / self.r_cmb
        return EMagOC(v[0], v[4], v[1], v[5], fos * v[8], fos * v[9], v[2], v[6], v[3], v[7],
                      0.0, 0.0)
