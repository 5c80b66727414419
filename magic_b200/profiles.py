"""Radial profiles for synthetic workloads (Boussinesq and anelastic).

Chebyshev-Gauss-Lobatto radii between r_icb = radratio/(1-radratio) and
r_cmb = 1/(1-radratio), outer boundary first (magic_torch/chebyshev.py), with
or2 = 1/r^2, or4 = 1/r^4, orho1 = orho2 = 1 (Boussinesq,
magic_torch/radial_functions.py:19-31) and the Courant spacings delxr2, delxh2
(magic_torch/radial_functions.py:190-197).
"""

import math

import torch


def boussinesq_profiles(n_r, l_max, radratio=0.35, device="cuda"):
    r_cmb = 1.0 / (1.0 - radratio)
    r_icb = r_cmb - 1.0
    k = torch.arange(n_r, dtype=torch.float64)
    r = r_icb + (r_cmb - r_icb) * 0.5 * (1.0 + torch.cos(math.pi * k / (n_r - 1)))
    dr = r[:-1] - r[1:]
    delxr2 = torch.empty(n_r, dtype=torch.float64)
    delxr2[0] = dr[0] ** 2
    delxr2[-1] = dr[-1] ** 2
    delxr2[1:-1] = torch.minimum(dr[:-1], dr[1:]) ** 2
    prof = dict(r=r, or2=1.0 / r ** 2, or4=1.0 / r ** 4, orho1=torch.ones(n_r, dtype=torch.float64),
                orho2=torch.ones(n_r, dtype=torch.float64), delxr2=delxr2,
                delxh2=r ** 2 / float(l_max * (l_max + 1)))
    return {k: v.to(device) for k, v in prof.items()}


def anelastic_profiles(n_r, l_max, radratio=0.35, strat=5.0, polind=2.0, device="cuda"):
    """Polytropic anelastic background on the same radii: temp0 = 1 + c (r_cmb/r - 1)
    with ``strat`` density scale heights across the shell, rho0 = temp0^polind,
    beta = d ln rho0/dr, otemp1 = 1/temp0, orho1 = 1/rho0, orho2 = orho1^2 (the
    polytropic background of magic_torch/radial_functions.py), unit viscosity and
    magnetic diffusivity."""
    p = boussinesq_profiles(n_r, l_max, radratio, device="cpu")
    r = p["r"]
    r_cmb = 1.0 / (1.0 - radratio)
    r_icb = r_cmb - 1.0
    c = (math.exp(strat / polind) - 1.0) / (r_cmb / r_icb - 1.0)
    temp0 = 1.0 + c * (r_cmb / r - 1.0)
    rho0 = temp0 ** polind
    beta = polind * (-c * r_cmb / r ** 2) / temp0
    p.update(or1=1.0 / r, beta=beta, otemp1=1.0 / temp0, orho1=1.0 / rho0,
             orho2=1.0 / rho0 ** 2, visc=torch.ones(n_r, dtype=torch.float64),
             lambda_=torch.ones(n_r, dtype=torch.float64))
    return {k: v.to(device) for k, v in p.items()}
