"""A run of the dynamo with the reference's run outputs (magic_torch/main.py:280-890).

- ``log.csv``: the columns step, sim_time, e_kin_pol, e_kin_tor, e_mag_pol,
  e_mag_tor, wall_elapsed, ms_per_step. A row is written at step 0 on a fresh
  start, every ``log_every`` steps, and at the last step.
- ``e_kin.<tag>`` / ``e_mag_oc.<tag>``: the Fortran-format energy lines of
  output.py:304-319. These are time then 8 (or 12) energies, in ES20.12 then
  ES16.8 fields.
- ``checkpoint_<step:06d>.pt``: written every ``checkpoint_every`` steps and
  at the last step, in the reference's checkpoint dictionary
  (magic_b200.state).

The step is any object with ``step()``, ``energies()`` and the state that
magic_b200.state reads (BoussinesqStep). Energies are computed on the GPU
and read back only at log steps.
"""

import csv
import os
import time

import torch

from .state import save_checkpoint

LOG_COLUMNS = ["step", "sim_time", "e_kin_pol", "e_kin_tor", "e_mag_pol", "e_mag_tor",
               "wall_elapsed", "ms_per_step"]


def write_e_kin_line(f, time_out, ek):
    """One e_kin.TAG line: ES20.12, 8 ES16.8 (output.py:304-309)."""
    f.write(f"{time_out:20.12E}" + "".join(f"{v:16.8E}" for v in (
        ek.e_p, ek.e_t, ek.e_p_as, ek.e_t_as, ek.e_p_es, ek.e_t_es, ek.e_p_eas, ek.e_t_eas))
        + "\n")


def write_e_mag_oc_line(f, time_out, em):
    """One e_mag_oc.TAG line: ES20.12, 12 ES16.8 (output.py:312-319)."""
    f.write(f"{time_out:20.12E}" + "".join(f"{v:16.8E}" for v in (
        em.e_p, em.e_t, em.e_p_as, em.e_t_as, em.e_p_os, em.e_p_as_os, em.e_p_es, em.e_t_es,
        em.e_p_eas, em.e_t_eas, em.e_p_e, em.e_p_as_e)) + "\n")


def run(st, n_steps, output_dir, tag="gpu", log_every=100, checkpoint_every=0, start_step=0,
        sim_time=0.0, cfg=None, t_scale=1.0, clock=time.perf_counter, adaptive=False):
    """Steps st from start_step + 1 to n_steps (main.py:843-886); returns sim_time.
    A restart (start_step > 0) appends to existing files and writes no step-0 row.
    adaptive: the Courant control of dt every step, as the reference's run loop."""
    os.makedirs(output_dir, exist_ok=True)
    mode = "a" if start_step > 0 else "w"
    log_path = os.path.join(output_dir, "log.csv")
    appending = start_step > 0 and os.path.exists(log_path)
    with open(log_path, "a" if appending else "w", newline="") as log_file, \
            open(os.path.join(output_dir, f"e_kin.{tag}"), mode) as f_ekin, \
            open(os.path.join(output_dir, f"e_mag_oc.{tag}"), mode) as f_emag:
        writer = csv.writer(log_file)
        if not appending:
            writer.writerow(LOG_COLUMNS)

        def write_row(step, t_sim, wall, steps_done):
            ek, em = st.energies()
            ms = wall / steps_done * 1000.0 if steps_done > 0 else 0.0
            writer.writerow([step, f"{t_sim:.10e}", f"{ek.e_p:.15e}", f"{ek.e_t:.15e}",
                             f"{em.e_p:.15e}", f"{em.e_t:.15e}", f"{wall:.3f}", f"{ms:.3f}"])
            log_file.flush()
            write_e_kin_line(f_ekin, t_sim * t_scale, ek)
            write_e_mag_oc_line(f_emag, t_sim * t_scale, em)
            f_ekin.flush()
            f_emag.flush()

        if start_step == 0:
            write_row(0, sim_time, 0.0, 0)
        t0 = clock()
        for n in range(start_step + 1, n_steps + 1):
            if adaptive:
                st.step(adaptive=True)
            else:
                st.step()
            sim_time += st.dt[0]
            if n % log_every == 0 or n == n_steps:
                if torch.cuda.is_available():
                    torch.cuda.synchronize()
                write_row(n, sim_time, clock() - t0, n - start_step)
            if checkpoint_every and (n % checkpoint_every == 0 or n == n_steps):
                save_checkpoint(st, os.path.join(output_dir, f"checkpoint_{n:06d}.pt"), step=n,
                                sim_time=sim_time, cfg=cfg)
    return sim_time
