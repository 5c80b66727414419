"""Radial profiles for synthetic workloads (Boussinesq and anelastic).

Chebyshev-Gauss-Lobatto radii between r_icb = radratio/(1-radratio) and
r_cmb = 1/(1-radratio), outer boundary first (magic_torch/chebyshev.py), with
or2 = 1/r^2, or4 = 1/r^4, orho1 = orho2 = 1 (Boussinesq,
magic_torch/radial_functions.py:19-31) and the Courant spacings delxr2, delxh2
(magic_torch/radial_functions.py:190-197).
"""

import math

import numpy as np
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


def polytropic_background(r, radratio=0.35, strat=5.0, polind=2.0, g0=0.0, g1=0.0, g2=1.0,
                          pr=1.0, ra=3e6, ek=1e-4, prmag=5.0, l_mag=False):
    """The anelastic polytropic reference state on radii ``r`` (numpy, FP64;
    magic_torch/radial_functions.py:70-165, radial.f90:622-764): gravity
    g0 + g1 r / r_cmb + g2 r_cmb^2 / r^2, dissipation number DissNb from ``strat``
    density scale heights, temp0, rho0 = temp0^polind, beta = d ln rho0 / dr and
    its derivatives, d ln temp0 / dr, 1/rho0, 1/rho0^2, 1/temp0, and the viscous
    and Ohmic heating factors (Ohmic only with a magnetic field).  Transport
    properties are constant (visc = kappa = lambda = 1), as in the reference."""
    r = np.asarray(r, dtype=np.float64)
    r_cmb = 1.0 / (1.0 - radratio)
    r_icb = r_cmb - 1.0
    or1 = 1.0 / r
    or2, or3 = or1 * or1, or1 ** 3
    or4 = or2 * or2
    rgrav = g0 + g1 * r / r_cmb + g2 * r_cmb ** 2 * or2
    diss = ((math.exp(strat / polind) - 1.0) / (r_cmb - r_icb)
            / (g0 + 0.5 * g1 * (1.0 + radratio) + g2 / radratio))
    temp0 = (-diss * (g0 * r + 0.5 * g1 * r ** 2 / r_cmb - g2 * r_cmb ** 2 * or1)
             + 1.0 + diss * r_cmb * (g0 + 0.5 * g1 - g2))
    rho0 = temp0 ** polind
    beta = -polind * diss * rgrav / temp0
    dgrav = g1 / r_cmb - 2.0 * g2 * r_cmb ** 2 * or3
    dbeta = -polind * diss / temp0 ** 2 * (dgrav * temp0 + diss * rgrav ** 2)
    ddbeta = -polind * diss / temp0 ** 3 * (
        temp0 * (6.0 * g2 * r_cmb ** 2 * or4 * temp0 + diss * rgrav * dgrav)
        + 2.0 * diss * rgrav * (diss * rgrav ** 2 + dgrav * temp0))
    dtemp0, d2temp0 = -diss * rgrav, -diss * dgrav
    visc_heat = diss * pr / ra
    return dict(rgrav=rgrav, temp0=temp0, rho0=rho0, beta=beta, dbeta=dbeta, ddbeta=ddbeta,
                dLtemp0=dtemp0 / temp0, ddLtemp0=-(dtemp0 / temp0) ** 2 + d2temp0 / temp0,
                orho1=1.0 / rho0, orho2=1.0 / rho0 ** 2, otemp1=1.0 / temp0, DissNb=diss,
                ViscHeatFac=visc_heat,
                OhmLossFac=visc_heat / (ek * prmag ** 2) if l_mag else 0.0)


def anelastic_profiles(n_r, l_max, radratio=0.35, strat=5.0, polind=2.0, device="cuda"):
    """The polytropic background (polytropic_background, gravity ~ 1/r^2) on the
    Chebyshev radii of boussinesq_profiles, with or1, unit viscosity and magnetic
    diffusivity, as torch tensors for the stage kernels."""
    p = boussinesq_profiles(n_r, l_max, radratio, device="cpu")
    r = p["r"]
    bg = polytropic_background(r.numpy(), radratio, strat, polind)
    t = lambda x: torch.as_tensor(x, dtype=torch.float64)
    p.update(or1=1.0 / r, beta=t(bg["beta"]), otemp1=t(bg["otemp1"]), orho1=t(bg["orho1"]),
             orho2=t(bg["orho2"]), visc=torch.ones(n_r, dtype=torch.float64),
             lambda_=torch.ones(n_r, dtype=torch.float64))
    return {k: v.to(device) for k, v in p.items()}
