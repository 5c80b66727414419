"""Simulation state in the reference's checkpoint format.

magic_torch/main.py:189-267 saves one ``torch.save`` dictionary per
checkpoint: ``step``, ``sim_time``, ``cfg``, ``tscheme_dt`` (dt of the current
and the previous step), ``fields.<name>`` for every spectral field
(``(lm_max, n_r)`` complex128), ``fields.omega_ic`` / ``fields.omega_ma``, and
for every time array ``dt.<name>.old`` / ``.impl`` ``(lm_max, n_r, 1)`` and
``.expl`` ``(lm_max, n_r, 2)`` (slot 0 the current explicit term, slot 1 the
previous one), plus the rotation-rate scalars ``dt.domega_{ic,ma}_dt.*``.
The same dictionary is written and read here for a BoussinesqStep, so a run
can be resumed by either implementation from the other's file.  Fields and
time arrays a step does not evolve (composition, the rotation rates; dp and
dpdt in the double-curl form) are written as zeros and ignored on load.
"""

import torch

FIELD_NAMES = ["w_LMloc", "dw_LMloc", "ddw_LMloc", "z_LMloc", "dz_LMloc", "p_LMloc",
               "dp_LMloc", "s_LMloc", "ds_LMloc", "xi_LMloc", "dxi_LMloc", "b_LMloc",
               "db_LMloc", "ddb_LMloc", "aj_LMloc", "dj_LMloc", "ddj_LMloc"]
DT_NAMES = ["dsdt", "dxidt", "dwdt", "dzdt", "dpdt", "dbdt", "djdt"]

# reference field name -> BoussinesqStep.f key
_FIELD_MAP = {"w_LMloc": "w", "dw_LMloc": "dw", "ddw_LMloc": "ddw", "z_LMloc": "z",
              "dz_LMloc": "dz", "p_LMloc": "p", "dp_LMloc": "dp", "s_LMloc": "s",
              "ds_LMloc": "ds",
              "b_LMloc": "b", "db_LMloc": "db", "ddb_LMloc": "ddb", "aj_LMloc": "aj",
              "dj_LMloc": "dj", "ddj_LMloc": "ddj"}
# reference time array -> BoussinesqStep.ta key
_DT_MAP = {"dsdt": "s", "dwdt": "w", "dzdt": "z", "dpdt": "p", "dbdt": "b", "djdt": "j"}


def state_dict(st, step=0, sim_time=0.0, cfg=None):
    """The reference's checkpoint dictionary of a BoussinesqStep, on the CPU."""
    cpu = lambda x: x.detach().to("cpu", copy=True)
    zero = torch.zeros(st.lm_max, st.n_r, dtype=torch.complex128)
    out = {"step": int(step), "sim_time": float(sim_time), "cfg": dict(cfg or {}),
           "tscheme_dt": torch.tensor(st.dt, dtype=torch.float64)}
    for name in FIELD_NAMES:
        k = _FIELD_MAP.get(name)
        out["fields." + name] = cpu(st.f[k]) if k in st.f else zero.clone()
    out["fields.omega_ic"] = 0.0
    out["fields.omega_ma"] = 0.0
    for name in DT_NAMES:
        e = _DT_MAP.get(name)
        if e not in st.ta:
            old = impl = zero[..., None].clone()
            expl = torch.zeros(st.lm_max, st.n_r, 2, dtype=torch.complex128)
        else:
            ta = st.ta[e]
            old, impl = cpu(ta["old"])[..., None], cpu(ta["impl"])[..., None]
            expl = torch.stack((cpu(ta["expl0"]), cpu(ta["expl1"])), dim=-1)
        out[f"dt.{name}.impl"], out[f"dt.{name}.expl"], out[f"dt.{name}.old"] = impl, expl, old
    for sname in ("domega_ic_dt", "domega_ma_dt"):
        out[f"dt.{sname}.impl"] = torch.zeros(1, dtype=torch.float64)
        out[f"dt.{sname}.expl"] = torch.zeros(2, dtype=torch.float64)
        out[f"dt.{sname}.old"] = torch.zeros(1, dtype=torch.float64)
    return out


def load_state_dict(st, state):
    """Fill a BoussinesqStep from a reference checkpoint dictionary (main.py:225-267):
    fields, time arrays, and the dt pair (new solve operators when it changed).
    Returns (step, sim_time)."""
    shape = (st.lm_max, st.n_r)
    for name, k in _FIELD_MAP.items():
        if k not in st.f:
            continue
        v = state["fields." + name]
        if tuple(v.shape) != shape:
            raise ValueError(f"fields.{name}: shape {tuple(v.shape)}, expected {shape}")
        st.f[k].copy_(v.to(st.device, torch.complex128))
    for name, e in _DT_MAP.items():
        if e not in st.ta:
            continue
        ta = st.ta[e]
        expl = state[f"dt.{name}.expl"]
        if tuple(expl.shape) != shape + (2,):
            raise ValueError(f"dt.{name}.expl: shape {tuple(expl.shape)}, expected {shape + (2,)}")
        ta["old"].copy_(state[f"dt.{name}.old"][..., 0].to(st.device, torch.complex128))
        ta["impl"].copy_(state[f"dt.{name}.impl"][..., 0].to(st.device, torch.complex128))
        ta["expl0"].copy_(expl[..., 0].to(st.device, torch.complex128))
        ta["expl1"].copy_(expl[..., 1].to(st.device, torch.complex128))
    if "tscheme_dt" in state:
        dt = state["tscheme_dt"]
        st.set_dt(float(dt[0]), float(dt[1]))
    return int(state.get("step", 0)), float(state.get("sim_time", 0.0))


def save_checkpoint(st, path, step=0, sim_time=0.0, cfg=None):
    """main.py:189-222: one torch.save dictionary."""
    torch.save(state_dict(st, step, sim_time, cfg), path)


def load_checkpoint(st, path):
    """main.py:225-267; returns (step, sim_time)."""
    return load_state_dict(st, torch.load(path, weights_only=False))
