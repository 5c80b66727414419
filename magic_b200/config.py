"""Configuration of the module-level, reference-signature API.

The reference reads its resolution and physics from module globals fixed at
import (``magic_torch/config.py:19-33``, ``magic_torch/params.py:56-202``).
This package keeps the same calling convention for ``magic_b200.sht`` and
``magic_b200.get_nl``: call ``configure({...})`` once (keys as in the
reference: ``l_max``, ``minc``, ``ek``, ``prmag``, ``device`` ...), or
``configure_from_reference()`` inside a process that already imported
``magic_torch`` so both agree on every size.  Plans are built lazily, one per
(l_max, minc, precision, device).
"""

import math

_config = {}
_plans = {}


def configure(overrides=None):
    """Replace the configuration (mirrors ``magic_torch.config.configure``)."""
    global _config
    _config = dict(overrides or {})


def get(key, default=None):
    return _config.get(key, default)


def configure_from_reference():
    """Copy resolution and radial profiles from an imported ``magic_torch``."""
    import sys

    if "magic_torch.params" not in sys.modules:
        raise RuntimeError("magic_torch is not imported in this process")
    import magic_torch.params as P
    import magic_torch.pre_calculations as pc
    import magic_torch.radial_functions as rf
    import magic_torch.radial_scheme as rs

    # get_nl_anel reads r from radial_scheme and ViscHeatFac / OhmLossFac from
    # radial_functions (magic_torch/get_nl_anel.py:14-16); courant_check reads
    # LFfac and opm (magic_torch/courant.py:12-14)
    cfg = dict(l_max=P.l_max, minc=P.minc, LFfac=float(pc.LFfac), opm=float(pc.opm),
               ViscHeatFac=float(rf.ViscHeatFac), OhmLossFac=float(rf.OhmLossFac),
               r=rs.r)
    for k in ("or1", "or2", "or4", "orho1", "orho2", "beta", "otemp1", "visc", "lambda_",
              "delxr2", "delxh2"):
        cfg[k] = getattr(rf, k)
    configure(cfg)


def lffac():
    if "LFfac" in _config:
        return float(_config["LFfac"])
    ek = float(_config.get("ek", 1e-3))
    prmag = float(_config.get("prmag", 5.0))
    return 1.0 / (ek * prmag)  # magic_torch/pre_calculations.py:27-28


def default_plan():
    from .plan import Plan
    import torch

    l_max = int(_config.get("l_max", 16))
    minc = int(_config.get("minc", 1))
    prec = str(_config.get("precision", "fp64"))
    dev = torch.device(_config.get("device", "cuda"))
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    key = (l_max, minc, prec, str(dev))
    if key not in _plans:
        _plans[key] = Plan(l_max, minc, precision=prec, device=dev)
    return _plans[key]


def profile(name, n_r):
    """A radial profile from the configuration, or the Boussinesq default."""
    import torch

    if name in _config:
        return torch.as_tensor(_config[name], dtype=torch.float64)
    if name in ("orho1", "orho2", "otemp1", "visc", "lambda_"):
        return torch.ones(n_r, dtype=torch.float64)
    if name == "beta":
        return torch.zeros(n_r, dtype=torch.float64)
    raise KeyError(f"radial profile {name!r} not configured")


__all__ = ["configure", "configure_from_reference", "default_plan", "get", "lffac", "profile",
           "math"]
