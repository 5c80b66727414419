"""A whole CNAB2 time step of the Boussinesq MHD dynamo on the GPU
(magic_b200.step.BoussinesqStep: fused nonlinear stage, explicit terms,
implicit solves S, Z, W, B), checked as a composition of the entry points
that the other GPU tests pin against the reference: repeated steps stay
finite and reproduce bit for bit, the split-precision and FP64 stages agree
to the split tolerance after a few steps, and without buoyancy or rotation
the kinetic and magnetic parts of a small perturbation only decay."""

import pytest
import torch

pytestmark = pytest.mark.gpu


def _energy(st):
    return sum(float((st.f[k].abs() ** 2).sum()) for k in ("w", "z", "b", "aj"))


def _run(precision, n, **kw):
    from magic_b200.step import BoussinesqStep

    st = BoussinesqStep(32, 33, precision=precision, **kw)
    st.init_random(seed=1, amp=1e-3)
    dts = []
    for _ in range(n):
        dts.append(st.step())
    torch.cuda.synchronize()
    return st, dts


def test_step_is_finite_and_deterministic():
    a, dts = _run("fp64", 3)
    b, _ = _run("fp64", 3)
    for k in a.f:
        assert torch.isfinite(torch.view_as_real(a.f[k])).all(), k
        assert torch.equal(a.f[k], b.f[k]), k
    assert all(torch.isfinite(d).all() for pair in dts for d in pair)


def test_split_stage_tracks_fp64_stage():
    a, _ = _run("fp64", 3)
    b, _ = _run("split", 3)
    for k in ("w", "z", "s", "b", "aj"):
        e = ((a.f[k] - b.f[k]).abs().max() / a.f[k].abs().max()).item()
        assert e < 1e-4, (k, e)


def test_pure_diffusion_decays():
    a, _ = _run("fp64", 1, ra=0.0, ek=1e6)
    e0 = _energy(a)
    for _ in range(5):
        a.step()
    torch.cuda.synchronize()
    assert _energy(a) < e0


# ---- against the reference's own time steps -------------------------------

STEP_FIELDS = ("w", "dw", "ddw", "z", "dz", "s", "ds", "b", "db", "ddb", "aj", "dj", "ddj")
STEP_DT = {"s": "dsdt", "z": "dzdt", "w": "dwdt", "b": "dbdt", "j": "djdt"}


def _golden_state(z, tag):
    import numpy as np

    return {k.split(":", 1)[1]: torch.as_tensor(np.ascontiguousarray(z[k]))
            for k in z if k.startswith(tag + ":") and "." in k.split(":", 1)[1]} | {
        "tscheme_dt": torch.as_tensor(z[tag + ":tscheme_dt"])}


def _reference_run(name="step_fd"):
    from conftest import load_golden
    from magic_b200.state import load_state_dict
    from magic_b200.step import BoussinesqStep

    z = load_golden(name)
    st = BoussinesqStep(int(z["l_max"]), int(z["n_r_max"]), ek=float(z["ek"]), ra=float(z["ra"]),
                        pr=float(z["pr"]), prmag=float(z["prmag"]), dt=float(z["dt"]),
                        precision="fp64", radratio=float(z["radratio"]), minc=int(z["minc"]),
                        radial_scheme="chebyshev" if "cheb" in name else "FD")
    assert st.lm_max == int(z["lm_max"])
    load_state_dict(st, _golden_state(z, "0"))
    return z, st


def test_two_steps_match_reference():
    """Two whole CNAB2 steps (FP64 stage) from the reference's own initial state
    (setup_initial_state after seeded perturbations of s, w and z) against the
    reference's one_step results (tests/golden/step_fd.npz, l_max = 12, 13 FD4
    levels, Ek 1e-3, Ra 1e5, Pm 5, dt 1e-4): every field the step evolves and
    every time array, and the kinetic / magnetic energies.  Tolerance, relative
    to each array's largest value: 1e-12 for the fields w, z, s, b, aj, the
    l = 0 pressure and the energies (measured <= 4.3e-14); 1e-11 for the radial
    derivatives and the time arrays (measured <= 1.5e-12 in the entropy's
    implicit term): they apply D2 (and D4 through the double curl) to the new
    fields of a state whose explicit terms reach 7e6."""
    import numpy as np

    z, st = _reference_run()
    rel = lambda a, b: float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    st.step()
    for k in ("w", "z", "s", "b", "aj"):
        e = rel(st.f[k].cpu().numpy(), z[f"1:fields.{k}_LMloc"])
        assert e < 1e-12, ("step 1", k, e)
    st.step()
    errs = {}
    for k in STEP_FIELDS:
        errs[k] = rel(st.f[k].cpu().numpy(), z[f"2:fields.{k}_LMloc"])
    errs["p00"] = rel(st.f["p"][0].cpu().numpy(), z["2:fields.p_LMloc"][0])
    for e, name in STEP_DT.items():
        ta = st.ta[e]
        errs[name + ".old"] = rel(ta["old"].cpu().numpy(), z[f"2:dt.{name}.old"][..., 0])
        errs[name + ".impl"] = rel(ta["impl"].cpu().numpy(), z[f"2:dt.{name}.impl"][..., 0])
        errs[name + ".expl0"] = rel(ta["expl0"].cpu().numpy(), z[f"2:dt.{name}.expl"][..., 0])
        errs[name + ".expl1"] = rel(ta["expl1"].cpu().numpy(), z[f"2:dt.{name}.expl"][..., 1])
    ek, em = st.energies()
    errs["e_kin"] = rel(np.array(ek), z["2:e_kin"])
    errs["e_mag"] = rel(np.array(em), z["2:e_mag"])
    print({k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        tight = k in ("w", "z", "s", "b", "aj", "p00", "e_kin", "e_mag")
        assert v < (1e-12 if tight else 1e-11), (k, v)


def test_two_steps_match_reference_chebyshev():
    """Two whole steps on Chebyshev levels with the standard (w, p) form from the
    reference's own initial state (tests/golden/step_cheb.npz: l_max 32, minc 4,
    33 levels, Ek 1e-3, Ra 1e5, Pm 5, dt 5e-6, seeded perturbations of s, w and
    z): the fields (p and dp included), every time array (dpdt included) and the
    energies against the reference's one_step results (its whole-step path, which
    stores the w and p implicit terms as zero at l = 0 and at the boundaries).
    Tolerance, relative to each array's largest value: 1e-12 for the fields and
    the energies (measured <= 4.5e-13, in w), 1e-9 for the radial derivatives and
    the time arrays (measured <= 2.0e-10, in ddb: the Chebyshev D2 at 33 levels
    amplifies the fields' rounding-level differences ~1e5-fold)."""
    import numpy as np

    z, st = _reference_run("step_cheb")
    rel = lambda a, b: float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    st.step()
    st.step()
    errs = {k: rel(st.f[k].cpu().numpy(), z[f"2:fields.{k}_LMloc"])
            for k in STEP_FIELDS + ("p", "dp")}
    for e, name in dict(STEP_DT, p="dpdt").items():
        ta = st.ta[e]
        errs[name + ".old"] = rel(ta["old"].cpu().numpy(), z[f"2:dt.{name}.old"][..., 0])
        errs[name + ".impl"] = rel(ta["impl"].cpu().numpy(), z[f"2:dt.{name}.impl"][..., 0])
        errs[name + ".expl0"] = rel(ta["expl0"].cpu().numpy(), z[f"2:dt.{name}.expl"][..., 0])
        errs[name + ".expl1"] = rel(ta["expl1"].cpu().numpy(), z[f"2:dt.{name}.expl"][..., 1])
    ek, em = st.energies()
    errs["e_kin"] = rel(np.array(ek), z["2:e_kin"])
    errs["e_mag"] = rel(np.array(em), z["2:e_mag"])
    print({k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        tight = k in ("w", "z", "s", "b", "aj", "p", "e_kin", "e_mag")
        assert v < (1e-12 if tight else 1e-9), (k, v)


def test_checkpoint_round_trip(tmp_path):
    """save_checkpoint writes the reference's dictionary (main.py:189-222: the same
    keys and shapes as the reference's own file) and load_checkpoint restores a
    state that steps on identically."""
    import json

    from conftest import load_golden
    from magic_b200.state import load_checkpoint, save_checkpoint

    z, st = _reference_run()
    st.step()
    path = tmp_path / "ck.pt"
    save_checkpoint(st, path, step=1, sim_time=1e-4, cfg={"l_max": 12})
    saved = torch.load(path, weights_only=False)
    layout = json.loads(str(load_golden("step_fd")["ckpt_layout"]))
    assert set(saved) == set(layout)
    for k, v in layout.items():
        if isinstance(v, list):
            assert list(saved[k].shape) == v, k
    _, other = _reference_run()
    assert load_checkpoint(other, path) == (1, 1e-4)
    st.step()
    other.step()
    for k in STEP_FIELDS:
        assert torch.equal(st.f[k], other.f[k]), k


def test_split_stage_drift_after_500_steps():
    """500 steps at l_max = 255 on 97 FD4 levels (Ek 1e-5, Ra 3e8, dt 2e-7, seeded
    perturbation 1e-4 (l+1)^-2) with the split and the FP64 stage from one state:
    the split run's fields stay within 2e-7 of the FP64 run's (largest value of
    each field; measured 9.4e-8, the 1e-7 target) and its total energies within
    1e-6 (measured 2.4e-7; the 1e-9 energy target is not met)."""
    from magic_b200.step import BoussinesqStep

    runs = []
    for prec in ("fp64", "split"):
        st = BoussinesqStep(255, 97, precision=prec)
        st.init_random(seed=0, amp=1e-4)
        runs.append(st)
    a, b = runs
    for _ in range(500):
        a.step()
        b.step()
    fe = {k: ((a.f[k] - b.f[k]).abs().max() / a.f[k].abs().max()).item()
          for k in ("w", "z", "s", "b", "aj")}
    ea, eb = a.energies(), b.energies()
    ee = max(abs(x - y) / abs(x) for x, y in zip(ea[0][:2] + ea[1][:2], eb[0][:2] + eb[1][:2]))
    print(fe, ee)
    assert max(fe.values()) < 2e-7, fe
    assert ee < 1e-6, ee


def test_run_outputs_and_restart(tmp_path):
    """magic_b200.run from the reference's initial state: the energies logged
    after two steps equal the reference's (its e_kin / e_mag_oc after two
    one_step calls, to 1e-12), and a run restarted from its step-2 checkpoint
    ends bit for bit where the uninterrupted run ends."""
    import csv

    import numpy as np

    from magic_b200.run import run
    from magic_b200.state import load_checkpoint

    z, st = _reference_run()
    run(st, 4, str(tmp_path / "a"), log_every=1, checkpoint_every=2)
    rows = list(csv.reader(open(tmp_path / "a" / "log.csv")))
    r2 = rows[3]
    assert int(r2[0]) == 2
    ek_ref, em_ref = z["2:e_kin"], z["2:e_mag"]
    assert abs(float(r2[2]) - ek_ref[0]) <= 1e-12 * abs(ek_ref[0])
    assert abs(float(r2[3]) - ek_ref[1]) <= 1e-12 * abs(ek_ref[1])
    assert abs(float(r2[4]) - em_ref[0]) <= 1e-12 * abs(em_ref[0])
    assert abs(float(r2[5]) - em_ref[1]) <= 1e-12 * abs(em_ref[1])
    line = open(tmp_path / "a" / "e_kin.gpu").read().splitlines()[2]
    vals = np.array([float(line[20 + 16 * i:36 + 16 * i]) for i in range(8)])
    assert np.abs(vals - ek_ref).max() <= 1e-7 * np.abs(ek_ref).max()   # ES16.8 digits
    _, other = _reference_run()
    step, t = load_checkpoint(other, tmp_path / "a" / "checkpoint_000002.pt")
    assert step == 2
    run(other, 4, str(tmp_path / "a"), log_every=1, start_step=2, sim_time=t)
    for k in STEP_FIELDS:
        assert torch.equal(st.f[k], other.f[k]), k


def _reference_run500(precision, name="run_fd_l32m4"):
    from conftest import load_golden
    from magic_b200.state import load_state_dict
    from magic_b200.step import BoussinesqStep

    z = load_golden(name)
    scheme = "chebyshev" if "cheb" in name else "FD"
    st = BoussinesqStep(int(z["l_max"]), int(z["n_r_max"]), ek=float(z["ek"]), ra=float(z["ra"]),
                        pr=float(z["pr"]), prmag=float(z["prmag"]), dt=float(z["dt"]),
                        precision=precision, radratio=float(z["radratio"]),
                        minc=int(z["minc"]), radial_scheme=scheme)
    assert st.lm_max == int(z["lm_max"])
    load_state_dict(st, _golden_state(z, "0"))
    return z, st


def _run500_errors(precision, name="run_fd_l32m4"):
    """Fields after 500 steps (relative to each field's largest value) and the
    kinetic / magnetic energies of every step (relative to each energy's largest
    value over the run) against the reference's 500 one_step calls.  The steps
    take the Courant control of dt, which, as in the reference's run, keeps dt at
    its maximum every step."""
    import numpy as np

    z, st = _reference_run500(precision, name)
    n = int(z["steps"])
    ek, em = [], []
    for _ in range(n):
        st.step(adaptive=True)
        assert st.dt == (float(z["dt"]), float(z["dt"])), st.dt
        a, b = st.energies()
        ek.append(np.array(a))
        em.append(np.array(b))
    ek, em = np.stack(ek), np.stack(em)
    rel = lambda a, b: float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    keys = ("w", "z", "s", "b", "aj") + (("p",) if st.std_form else ())
    fe = {k: rel(st.f[k].cpu().numpy(), z[f"{n}:{k}"]) for k in keys}
    ee = {}
    growth = np.abs(ek[:, 0] - z["e_kin"][:, 0]) / np.abs(z["e_kin"][:, 0])
    print("e_kin relative error at steps 1, 10, 100, 250, 500:",
          [f"{growth[i]:.1e}" for i in (0, 9, 99, 249, 499)])
    for name, got, ref in (("e_kin", ek, z["e_kin"]), ("e_mag", em, z["e_mag"])):
        for c in range(ref.shape[1]):
            if np.abs(ref[:, c]).max() > 0:
                ee[f"{name}[{c}]"] = rel(got[:, c], ref[:, c])
    return fe, ee


def test_500_steps_match_reference_fp64():
    """500 CNAB2 steps with the FP64 stage from the reference's own initial state
    (tests/golden/run_fd_l32m4.npz, made by running the reference: l_max 32,
    minc 4, 33 FD4 levels, Ek 1e-3, Ra 1e5, Pr 1, Pm 5, dt 1e-4, its l = m = 4
    entropy mode of amplitude 0.1 and dipolar field, seeded entropy noise 1e-5).
    The fields after step 500 and the kinetic and magnetic energies of every step
    match the reference's to 1e-12 relative (measured: fields <= 4.8e-13, in z;
    energies <= 6.2e-14)."""
    fe, ee = _run500_errors("fp64")
    print({k: f"{v:.1e}" for k, v in (fe | ee).items()})
    assert max(fe.values()) < 1e-12, fe
    assert max(ee.values()) < 1e-12, ee


def test_500_steps_match_reference_split():
    """The same 500 steps with the split-precision stage (bf16x3 tensor-core
    Legendre contractions, FP32 phi stage; implicit solves, explicit terms and
    energies in FP64) against the reference's FP64 run.  Measured: fields 8e-8
    (s) to 8.9e-6 (z), energies 8e-8 to 1.3e-6; the bounds are 3e-5 and 5e-6.
    This misses the 1e-7 (fields) and 1e-9 (energies) targets: the nonlinear
    terms carry the FP32 phi stage's ~1e-7-1e-6 relative error every step, and
    the convecting flow (kinetic energy 0.44 -> 73 over the run) amplifies it."""
    fe, ee = _run500_errors("split")
    print({k: f"{v:.1e}" for k, v in (fe | ee).items()})
    assert max(fe.values()) < 3e-5, fe
    assert max(ee.values()) < 5e-6, ee


def test_500_steps_match_reference_chebyshev_fp64():
    """The shell case as the reference runs it (tests/golden/run_cheb_l32m4.npz:
    l_max 32, minc 4, 33 Chebyshev levels with the standard (w, p) form, Ek 1e-3,
    Ra 1e5, Pr 1, Pm 5, dt 1e-4, the reference's initial fields and seeded entropy
    noise 1e-5): 500 FP64 steps; the energies of every step within 1e-12 of the
    reference's (measured <= 5.5e-13) and the fields (p included) after step 500
    within 1e-11 (measured: z 4.4e-12, the others <= 7.3e-13).  The z figure
    misses the 1e-12 target: the Chebyshev D2 turns the two implementations'
    rounding-level differences into ~1e-10 relative differences of the
    derivatives every step (two-step test), and the convecting flow carries them
    into the fields.  For scale, the reference itself with its fields (not their
    derivatives) perturbed by 1e-16 (relative) after every step ends 8.9e-14
    away in z: the larger part of the difference enters through the derivative
    arrays."""
    fe, ee = _run500_errors("fp64", "run_cheb_l32m4")
    print({k: f"{v:.1e}" for k, v in (fe | ee).items()})
    assert max(fe.values()) < 1e-11, fe
    assert max(ee.values()) < 1e-12, ee


def test_500_steps_match_reference_chebyshev_split():
    """The same Chebyshev run with the split-precision stage against the
    reference's FP64 run (bounds as for the finite-difference run)."""
    fe, ee = _run500_errors("split", "run_cheb_l32m4")
    print({k: f"{v:.1e}" for k, v in (fe | ee).items()})
    assert max(fe.values()) < 3e-5, fe
    assert max(ee.values()) < 5e-6, ee


def test_500_steps_match_reference_ozaki():
    """The same 500 finite-difference steps with the digit-split (ozaki) stage:
    int8 digit planes on the tcgen05 integer pipe with exact accumulation and an
    FP64 phi stage.  Bounds: the north star's 1e-7 on the fields and 1e-9 on the
    energies of every step, against the reference's FP64 run."""
    fe, ee = _run500_errors("ozaki")
    print({k: f"{v:.1e}" for k, v in (fe | ee).items()})
    assert max(fe.values()) < 1e-7, fe
    assert max(ee.values()) < 1e-9, ee


def test_500_steps_match_reference_chebyshev_ozaki():
    """The Chebyshev run with the digit-split stage (bounds 1e-7 and 1e-9)."""
    fe, ee = _run500_errors("ozaki", "run_cheb_l32m4")
    print({k: f"{v:.1e}" for k, v in (fe | ee).items()})
    assert max(fe.values()) < 1e-7, fe
    assert max(ee.values()) < 1e-9, ee


def test_ozaki_stage_drift_after_500_steps():
    """500 steps at l_max = 255 on 97 FD4 levels with the digit-split and the FP64
    stage from one seeded state: fields within 1e-7 and total energies within
    1e-9 of the FP64-stage run."""
    from magic_b200.step import BoussinesqStep

    runs = []
    for prec in ("fp64", "ozaki"):
        st = BoussinesqStep(255, 97, precision=prec)
        st.init_random(seed=0, amp=1e-4)
        runs.append(st)
    a, b = runs
    for _ in range(500):
        a.step()
        b.step()
    b.plan.poll_status(block=True)
    fe = {k: ((a.f[k] - b.f[k]).abs().max() / a.f[k].abs().max()).item()
          for k in ("w", "z", "s", "b", "aj")}
    ea, eb = a.energies(), b.energies()
    ee = max(abs(x - y) / abs(x) for x, y in zip(ea[0][:2] + ea[1][:2], eb[0][:2] + eb[1][:2]))
    print(fe, ee)
    assert max(fe.values()) < 1e-7, fe
    assert ee < 1e-9, ee


def test_courant_dt_control_matches_reference():
    """Steps with the reference's Courant control of dt (step(adaptive=True)) from
    the reference's own initial state (tests/golden/adapt_cheb.npz: l_max 32,
    minc 4, 33 Chebyshev levels, dtmax 1e-4, seeded perturbations of s, w and z
    of 1e-3): over 30 steps the reference cuts dt to 6.8e-6 at step 1, raises it
    to 4.1e-5, 8.8e-5 and back to dtmax, rebuilding its matrices each time.  The
    GPU takes the same dt at every step (to 1e-12 relative; measured 7.1e-14, the
    Courant limits' rounding), and its energies after every step and its fields
    after the last stay within 1e-11 of the reference's (measured: energies
    2.3e-13, fields 1.5e-12 in z)."""
    import numpy as np

    from conftest import load_golden
    from magic_b200.state import load_state_dict
    from magic_b200.step import BoussinesqStep

    z = load_golden("adapt_cheb")
    st = BoussinesqStep(int(z["l_max"]), int(z["n_r_max"]), ek=float(z["ek"]), ra=float(z["ra"]),
                        pr=float(z["pr"]), prmag=float(z["prmag"]), dt=float(z["dtmax"]),
                        precision="fp64", radratio=float(z["radratio"]), minc=int(z["minc"]),
                        radial_scheme="chebyshev")
    load_state_dict(st, _golden_state(z, "0"))
    dts, ek, em = [], [], []
    for _ in range(int(z["steps"])):
        st.step(adaptive=True)
        dts.append(st.dt[0])
        a, b = st.energies()
        ek.append(np.array(a))
        em.append(np.array(b))
    rel = lambda a, b: float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    errs = {"dt": float(np.max(np.abs(np.array(dts) - z["dt"]) / z["dt"]))}
    errs |= {k: rel(st.f[k].cpu().numpy(), z[f"{int(z['steps'])}:{k}"])
             for k in ("w", "z", "s", "b", "aj", "p")}
    errs["e_kin"] = max(rel(np.stack(ek)[:, c], z["e_kin"][:, c]) for c in range(8))
    errs["e_mag"] = max(rel(np.stack(em)[:, c], z["e_mag"][:, c]) for c in range(10))
    print({k: f"{v:.1e}" for k, v in errs.items()})
    assert errs["dt"] < 1e-12, (dts, z["dt"])
    for k, v in errs.items():
        assert v < 1e-11, (k, v)
