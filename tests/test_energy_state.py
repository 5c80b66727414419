"""CPU checks of the energy oracle, the radial integration rules and the
checkpoint layout, against the reference's own outputs
(tests/golden/energy_*.npz, step_fd.npz)."""

import json
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import energy as oe


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", ["energy_cheb", "energy_fd"])
def test_energy_oracle_matches_reference(name):
    z = load_golden(name)
    N = int(z["n_r_max"])
    w = oe.cheb_weights(N, float(z["radratio"])) if z["chebyshev"] else oe.simps_weights(z["r"])
    assert np.abs(w - z["rint_w"]).max() < 1e-15
    ek = oe.e_kin_full(z["in_w"], z["in_dw"], z["in_z"], z["lm2l"], z["lm2m"], z["or2"],
                       z["orho1"], w)
    em = oe.e_mag_oc_full(z["in_b"], z["in_db"], z["in_aj"], z["lm2l"], z["lm2m"], z["or2"],
                          float(z["LFfac"]), z["r"][0], w)
    assert _rel(ek, z["e_kin"]) < 1e-15 and _rel(em, z["e_mag"]) < 1e-15


@pytest.mark.parametrize("name", ["energy_cheb", "energy_fd"])
def test_rint_weights_match_reference(name):
    from magic_b200.radial import clenshaw_curtis_weights, simpson_weights

    z = load_golden(name)
    N = int(z["n_r_max"])
    if z["chebyshev"]:
        w = clenshaw_curtis_weights(N, float(z["radratio"]), np.sqrt(2.0 / (N - 1)), 0.5)
    else:
        w = simpson_weights(z["r"])
    assert np.abs(w - z["rint_w"]).max() < 1e-15


def test_energy_oracle_on_reference_steps():
    """Energies of the reference's states before and after two steps."""
    from magic_b200.radial import fd_grid

    z = load_golden("step_fd")
    N = int(z["n_r_max"])
    r = fd_grid(N, float(z["radratio"]), 0.3, 0.1)
    w = oe.simps_weights(r)
    LFfac = 1.0 / (float(z["ek"]) * float(z["prmag"]))
    for tag in ("0", "2"):
        g = lambda k: z[f"{tag}:fields.{k}_LMloc"]
        ek = oe.e_kin_full(g("w"), g("dw"), g("z"), z["lm2l"], z["lm2m"], 1.0 / r ** 2,
                           np.ones(N), w)
        em = oe.e_mag_oc_full(g("b"), g("db"), g("aj"), z["lm2l"], z["lm2m"], 1.0 / r ** 2,
                              LFfac, r[0], w)
        assert _rel(ek, z[tag + ":e_kin"]) < 1e-15
        assert _rel(em, z[tag + ":e_mag"]) < 1e-15


def test_checkpoint_layout_matches_reference():
    """state_dict of a (host-side stand-in) step has the reference checkpoint's
    keys, shapes and scalar types (magic_torch/main.py:189-222)."""
    from magic_b200.state import state_dict

    z = load_golden("step_fd")
    lm, N = int(z["lm_max"]), int(z["n_r_max"])
    zero = lambda: torch.zeros(lm, N, dtype=torch.complex128)
    st = SimpleNamespace(
        lm_max=lm, n_r=N, dt=(1e-4, 1e-4),
        f={k: zero() for k in ("w", "dw", "ddw", "z", "dz", "s", "ds", "b", "db", "ddb", "aj",
                               "dj", "ddj", "p")},
        ta={e: {k: zero() for k in ("old", "impl", "expl0", "expl1")}
            for e in ("s", "z", "w", "b", "j")})
    d = state_dict(st, step=3, sim_time=0.5, cfg={"l_max": 12})
    layout = json.loads(str(z["ckpt_layout"]))
    assert set(d) == set(layout)
    for k, v in layout.items():
        if isinstance(v, list):
            assert list(d[k].shape) == v, k
        else:
            assert type(d[k]).__name__ == v, k


class _FakeStep:
    """Host-side stand-in with the state layout of BoussinesqStep."""

    def __init__(self, lm=6, n_r=5):
        from collections import namedtuple

        from magic_b200.output import EKin, EMagOC

        self.lm_max, self.n_r, self.dt, self.count = lm, n_r, (1e-4, 1e-4), 0
        self.device = torch.device("cpu")
        z = lambda: torch.zeros(lm, n_r, dtype=torch.complex128)
        self.f = {k: z() for k in ("w", "dw", "ddw", "z", "dz", "s", "ds", "b", "db", "ddb",
                                   "aj", "dj", "ddj", "p")}
        self.ta = {e: {k: z() for k in ("old", "impl", "expl0", "expl1")}
                   for e in ("s", "z", "w", "b", "j")}
        self._EKin, self._EMag = EKin, EMagOC

    def step(self):
        self.count += 1
        self.f["w"] += 1.0

    def energies(self):
        c = float(self.count)
        return (self._EKin(*[c + 0.125 * i for i in range(8)]),
                self._EMag(*[-c - 0.25 * i for i in range(12)]))

    def set_dt(self, a, b):
        self.dt = (a, b)


def test_run_outputs_follow_the_reference_layout(tmp_path):
    """log.csv columns and cadence, Fortran-format energy lines and checkpoint
    names of magic_torch/main.py:385-886 and output.py:304-319."""
    import csv

    from magic_b200.run import LOG_COLUMNS, run
    from magic_b200.state import load_state_dict

    st = _FakeStep()
    t = run(st, 7, str(tmp_path), tag="x", log_every=3, checkpoint_every=4)
    assert t == pytest.approx(7e-4)
    rows = list(csv.reader(open(tmp_path / "log.csv")))
    assert rows[0] == LOG_COLUMNS
    assert [int(r[0]) for r in rows[1:]] == [0, 3, 6, 7]
    assert float(rows[2][2]) == 3.0 and float(rows[2][4]) == -3.0
    ek = open(tmp_path / "e_kin.x").read().splitlines()
    em = open(tmp_path / "e_mag_oc.x").read().splitlines()
    assert len(ek) == 4 and all(len(x) == 20 + 8 * 16 for x in ek)
    assert len(em) == 4 and all(len(x) == 20 + 12 * 16 for x in em)
    assert float(ek[1][:20]) == pytest.approx(3e-4) and float(ek[1][20:36]) == 3.0
    assert sorted(p.name for p in tmp_path.glob("checkpoint_*.pt")) == [
        "checkpoint_000004.pt", "checkpoint_000007.pt"]
    other = _FakeStep()
    assert load_state_dict(other, torch.load(tmp_path / "checkpoint_000004.pt",
                                             weights_only=False)) == (4, pytest.approx(4e-4))
    assert torch.equal(other.f["w"], torch.full_like(other.f["w"], 4.0))
    # a restart appends: no new header, no step-0 row
    run(other, 9, str(tmp_path), tag="x", log_every=3, start_step=4, sim_time=4e-4)
    rows = list(csv.reader(open(tmp_path / "log.csv")))
    assert [r[0] for r in rows].count("step") == 1
    assert [int(r[0]) for r in rows[1:]] == [0, 3, 6, 7, 6, 9]


def test_dt_courant_matches_oracle_and_reference_sequence():
    """The time step's Courant control (magic_b200.step.dt_courant) takes the same
    branch and value as the oracle's restatement of courant.py:130-155 on every
    regime (above dt_max, above the limit, far below it, in the keep band), and
    replays the reference's own dt sequence of tests/golden/adapt_cheb.npz: each
    decision from the previous dt and dtmax lands on the reference's next dt when
    fed the limit that decision implies (dt_min = dt_new / 0.75)."""
    import numpy as np

    from conftest import load_golden
    from magic_b200.step import dt_courant
    from oracle.nonlinear import dt_courant as ref_dt_courant

    cases = [(2e-4, 1e-4, 5e-4), (1e-4, 1e-4, 5e-5), (1e-6, 1e-4, 5e-5), (1e-5, 1e-4, 1.5e-5),
             (1e-4, 1e-4, 1e-3), (4e-5, 1e-4, 6e-5)]
    for dt, dtmax, dmin in cases:
        assert dt_courant(dt, dtmax, dmin) == ref_dt_courant(dt, dtmax, dmin, dmin), (dt, dmin)
    z = load_golden("adapt_cheb")
    dts, dtmax = [float(x) for x in z["dt"]], float(z["dtmax"])
    prev = dtmax
    for d in dts:
        if d != prev and d < dtmax:
            changed, new = dt_courant(prev, dtmax, d / 0.75)
            assert changed and abs(new - d) <= 1e-15 * d, (prev, d, new)
        prev = d
