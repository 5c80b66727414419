"""Reference-signature grid-space nonlinear terms and Courant check.

Drop-in for ``magic_torch.get_nl.get_nl`` (get_nl.py:30-87),
``magic_torch.get_nl_anel.get_nl_anel`` (get_nl_anel.py:41-136) and
``magic_torch.courant.courant_check`` (courant.py:80-127).  The reference
takes radial profiles from module globals; here they come from
``magic_b200.config`` unless passed.
"""

from . import config
from .config import default_plan


def get_nl(vrc, vtc, vpc, cvrc, cvtc, cvpc, sc, brc, btc, bpc, cbrc, cbtc, cbpc, xic,
           or4_3=None, or2_3=None, LFfac=None):
    n_r = vrc.shape[0]
    or4 = or4_3 if or4_3 is not None else config.profile("or4", n_r)
    or2 = or2_3 if or2_3 is not None else config.profile("or2", n_r)
    return default_plan().get_nl([vrc, vtc, vpc, cvrc, cvtc, cvpc, sc, brc, btc, bpc, cbrc, cbtc,
                                  cbpc, xic], or2, or4, config.lffac() if LFfac is None else LFfac)


def get_nl_anel(vrc, vtc, vpc, dvrdrc, dvtdrc, dvpdrc, dvrdtc, dvrdpc, dvtdpc, dvpdpc, cvrc,
                sc, xic, brc, btc, bpc, cbrc, cbtc, cbpc, prof=None, LFfac=None,
                ViscHeatFac=None, OhmLossFac=None, l_mag=True):
    n_r = vrc.shape[0]
    names = ("r", "or1", "or2", "or4", "beta", "orho1", "otemp1", "visc", "lambda_")
    prof = dict(prof or {})
    for k in names:
        if k not in prof:
            prof[k] = config.profile(k, n_r)
    return default_plan().get_nl_anel(
        [vrc, vtc, vpc, dvrdrc, dvtdrc, dvpdrc, dvrdtc, dvrdpc, dvtdpc, dvpdpc, cvrc, sc, xic,
         brc, btc, bpc, cbrc, cbtc, cbpc], prof,
        config.lffac() if LFfac is None else LFfac,
        float(config.get("ViscHeatFac", 0.0)) if ViscHeatFac is None else ViscHeatFac,
        float(config.get("OhmLossFac", 0.0)) if OhmLossFac is None else OhmLossFac, l_mag)


def courant_check(vrc, vtc, vpc, brc=None, btc=None, bpc=None, courfac=2.5, alffac=1.0,
                  prof=None, damp=True):
    n_r = vrc.shape[0]
    prof = dict(prof or {})
    for k in ("or2", "or4", "orho1", "orho2", "delxr2", "delxh2"):
        if k not in prof:
            prof[k] = config.profile(k, n_r)
    opm = float(config.get("opm", 1.0 / float(config.get("prmag", 5.0))))
    return default_plan().courant(vrc, vtc, vpc, brc, btc, bpc, prof, courfac, alffac,
                                  config.lffac(), opm, damp=damp)
