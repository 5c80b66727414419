"""Energy integrals on the GPU (mt_energy, FP64) against the reference's own
get_e_kin_full / get_e_mag_oc_full outputs (tests/golden/energy_*.npz:
Chebyshev points with minc = 2, and a fourth-order finite-difference grid
with an anelastic density profile) and against the oracle at l_max = 255 on
97 levels.  Tolerance 1e-13 of the largest component (FP64 sums in a
different order than the reference's)."""

import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import energy as oe

pytestmark = pytest.mark.gpu

TOL = 1e-13
cu = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", ["energy_cheb", "energy_fd"])
def test_energies_match_reference(name):
    from magic_b200 import Plan
    from magic_b200.output import EnergyIntegrals

    z = load_golden(name)
    p = Plan(int(z["l_max"]), int(z["minc"]))
    assert p.lm_max == int(z["lm_max"])
    E = EnergyIntegrals(p, z["r"], z["or2"], z["orho1"], z["rint_w"], float(z["LFfac"]))
    ek = E.kin(cu(z["in_w"]), cu(z["in_dw"]), cu(z["in_z"]))
    em = E.mag(cu(z["in_b"]), cu(z["in_db"]), cu(z["in_aj"]))
    print(name, _rel(ek, z["e_kin"]), _rel(em, z["e_mag"]))
    assert _rel(ek, z["e_kin"]) < TOL
    assert _rel(em, z["e_mag"]) < TOL


def test_energies_vs_oracle_l255():
    """l_max = 255, 97 FD4 levels, seeded spectra, an anelastic density profile."""
    from magic_b200 import Plan
    from magic_b200.output import EnergyIntegrals
    from magic_b200.radial import RadialScheme

    p = Plan(255, 1)
    sch = RadialScheme(97, "FD", fd_order=4)
    r = sch.r
    orho1 = np.exp(-0.4 * (r[0] - r))
    rng = np.random.default_rng(4)
    amp = (p.lm2l + 1.0)[:, None] ** -1.5
    spec = lambda: (rng.standard_normal((p.lm_max, 97))
                    + 1j * rng.standard_normal((p.lm_max, 97))) * amp
    f = {k: spec() for k in ("w", "dw", "z", "b", "db", "aj")}
    E = EnergyIntegrals(p, r, 1.0 / r ** 2, orho1, sch.rint, 200.0)
    ek = E.kin(cu(f["w"]), cu(f["dw"]), cu(f["z"]))
    em = E.mag(cu(f["b"]), cu(f["db"]), cu(f["aj"]))
    rint = oe.simps_weights(r)
    rk = oe.e_kin_full(f["w"], f["dw"], f["z"], p.lm2l, p.lm2m, 1.0 / r ** 2, orho1, rint)
    rm = oe.e_mag_oc_full(f["b"], f["db"], f["aj"], p.lm2l, p.lm2m, 1.0 / r ** 2, 200.0, r[0],
                          rint)
    assert _rel(ek, rk) < TOL and _rel(em, rm) < TOL
