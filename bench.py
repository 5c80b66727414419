"""Benchmark: whole CNAB2 time steps of the Boussinesq MHD dynamo at l_max=255 on B200.

One step = the reference's one_step (magic_torch/step_time.py:1574-1640): the
radial loop (Legendre synthesis of 13 grid fields on all 97 levels, the fused
phi-FFT + get_nl products + Courant kernel, the Legendre analysis of the 8
spectral outputs on the 95 bulk levels, then the explicit terms get_td +
finish_exp) and the lm loop (implicit CNAB2 solves of S, Z, W with the l = 0
pressure, B and J), at l_max = 255 (n_theta = 384, n_phi = 768, minc = 1) on 97
fourth-order finite-difference levels with the double-curl poloidal form
(Ek 1e-5, Ra 3e8, Pr = Pm = 1, dt 2e-7).  Seeded synthetic initial fields
(|c_lm| ~ 1e-4 (l+1)^-2); the spectral state (1.7 GB) is larger than L2.
The plain FP64 path (FP64 stage, same solves) is timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload step|stage|sht|anel|td|serve]

Under torchrun (N > 1) each rank runs an independent replica of the workload
(the step has no cross-GPU exchange); value = total steps/s over all ranks.
"""

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L_MAX, N_R = 255, 97
METRIC = "steps/s @lmax=255 vs FP64 plain, 1 B200; SHT TFLOP/s; ensemble p99 latency"
FIELDS = ("w", "dw", "ddw", "z", "dz", "s", "b", "db", "ddb", "aj", "dj")
OUTS = ("Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt", "VxBp")
LF, CF, AF, OPM = 1.0 / (1e-5 * 1.0), 2.5, 1.0, 1.0  # Ek=1e-5, Pm=1


def workload_config(prec):
    return {"workload": f"Boussinesq MHD radial-loop nonlinear stage ({prec})",
            "l_max": L_MAX, "minc": 1, "n_theta": 384, "n_phi": 768, "n_r": N_R,
            "grid_fields_in": 13, "spectral_out": 8, "l2": "inputs larger than L2 (561 MB)",
            "parallelism": "replicas"}


def flops_per_step(nhs, lm_max, n_r):
    """Algorithmic Legendre flops (convention: F = 4 NHS lm_max per scalar-equivalent
    contraction per level; torpol synthesis 3F, scalar 1F, vector analysis 4F)."""
    F = 4.0 * nhs * lm_max
    synth = n_r * (1 + 4 * 3) * F          # s + 4 torpol groups
    anal = (n_r - 2) * (3 * 1 + 3 * 4) * F  # Advr VSr VxBr + 3 vector pairs
    return synth, anal


def split_mma_flops(plan, n_r):
    """Dense bf16 tensor-pipe FLOPs the split kernels issue per step (6 plane products
    per table per 16-wide K chunk, M = 128 rows per CTA, padded tiles included)."""
    nhs = plan.nhs
    nth = 1 if nhs <= 256 else 2
    wth = (((nhs + nth - 1) // nth) + 15) // 16 * 16
    rows_s = n_r * 2 * 13
    rows_a = (n_r - 2) * 2 * 8
    tiles_s = -(-rows_s // 128)
    tiles_a = -(-rows_a // 128)
    syn = ana = 0.0
    nchj = -(-nhs // 16)
    for mc in range(plan.n_m_max):
        nlm = plan.l_max - mc * plan.minc + 1
        nk = [(nlm + 1) // 2, nlm // 2]
        nch = [-(-k // 16) for k in nk]
        for combo in (0, 1):
            chunks = nch[combo] + nch[1 - combo]  # P chunks + dP chunks
            syn += tiles_s * nth * chunks * 6 * 2.0 * 128 * wth * 16
        for par in (0, 1):
            wk = (nk[par] + 15) // 16 * 16
            ana += tiles_a * nchj * 2 * 6 * 2.0 * 128 * wk * 16
    return syn, ana


def ozaki_mma_ops(plan, n_r, nfi=13, nfo=9):
    """Dense int8 tensor-pipe operations the digit-split kernels issue per stage:
    21 digit-pair products per K chunk of 32 (issued as eight or six MMAs with the table
    planes stacked along N), M = 128 rows per tile, N = 64 theta rows
    (synthesis) or 32 l rows (analysis), padded tiles included."""
    kk, rows = 32, 128
    nhs = plan.nhs
    nthtile = -(-nhs // 64)
    tiles_s = -(-(n_r * 2 * nfi) // rows)
    lev_tile = rows // (2 * nfo)
    tiles_a = -(-(n_r - 2) // lev_tile)
    nchj = -(-nhs // kk)
    nk = lambda nlm, p: (nlm + 1 - p) // 2
    syn = ana = 0.0
    for mc in range(plan.n_m_max):
        nlm = plan.l_max - mc * plan.minc + 1
        for combo in (0, 1):
            steps = -(-nk(nlm, combo) // kk) + -(-nk(nlm, 1 - combo) // kk)
            syn += tiles_s * nthtile * steps * 21 * 2.0 * rows * 64 * kk
        for par in (0, 1):
            nlt = -(-nk(nlm, par) // 32)
            ana += tiles_a * nlt * nchj * 2 * 21 * 2.0 * rows * 32 * kk
    return syn, ana


def synth_inputs(plan, n_r, device, seed=0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    l = torch.as_tensor(plan.lm2l, dtype=torch.float64)
    m0 = torch.as_tensor(plan.lm2m == 0)
    amp = 1e-4 * (l + 1.0) ** -2
    out = {}
    for k in FIELDS:
        ph = torch.rand(plan.lm_max, n_r, generator=g, dtype=torch.float64) * 2 * math.pi
        mag = amp[:, None] * (0.5 + torch.rand(plan.lm_max, n_r, generator=g, dtype=torch.float64))
        c = torch.polar(mag, ph)
        c[m0] = c[m0].real.to(c.dtype)
        out[k] = c.to(device)
    return out


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML every
    10 ms while the timed region runs (reads only; nothing is set)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.max_mhz = None
        self.stop = threading.Event()
        self.started = threading.Event()
        self.nvml = None

    def _handle(self):
        import pynvml

        pynvml.nvmlInit()
        self.nvml = pynvml
        try:
            idx = torch.cuda._get_nvml_device_index(self.device)
        except Exception:
            idx = self.device.index or 0
        return pynvml.nvmlDeviceGetHandleByIndex(idx)

    def _run(self):
        try:
            h = self._handle()
            nv = self.nvml
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            reasons_fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            while True:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                     reasons_fn(h)))
                self.started.set()
                if self.stop.wait(0.01):
                    break
        except Exception as e:  # no NVML: the line says so
            self.error = repr(e)
        finally:
            self.started.set()

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        self.started.wait(10.0)
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(10.0)
        if self.nvml is not None:
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0,
                    "source": getattr(self, "error", "nvml")}
        reasons = sorted({n for _, r in self.samples for n, bit in self.REASONS.items()
                          if r & bit})
        sm = [c for c, _ in self.samples]
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm), "source": "nvml, 10 ms"}


# DRAM bytes (read + write) of one launch of the phi-stage kernel from an ncu
# full-set capture of the same kernel at l_max = 255, n_r = 17, per Fourier row moved (13 fields x n_r in, 9 fields x (n_r - 2) out); traffic grows
# in proportion to the rows, so the full-size launch is scaled by its row count.
NCU_PHI_TRAFFIC = {"split": (230.161408e6 + 104.267520e6) / (13 * 17 + 9 * 15),
                   # the FP64 phi kernel of the digit-split stage (k_nl_bouss_w64)
                   "ozaki": (347.744000e6 + 178.849280e6) / (13 * 17 + 9 * 15)}
# warp instructions of the same launch (smsp__inst_executed.sum), per Fourier row
NCU_PHI_INST = {"split": 184287744.0 / (13 * 17 + 9 * 15),
                "ozaki": 209674368.0 / (13 * 17 + 9 * 15)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d, "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, \
            "fallback"


def dgemm_peak(device):
    """cuBLAS FP64 DGEMM throughput (TFLOP/s), the FP64 tensor-pipe denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def cpu_stage_sample(n_levels=5, seed=0):
    """Time the CPU restatement (oracle) of the same stage on a bounded sample."""
    import numpy as np

    from oracle import fast as ofast

    t0 = time.perf_counter()
    g = ofast.FastGrid(L_MAX)
    build_s = time.perf_counter() - t0
    rng = np.random.default_rng(seed)
    amp = 1e-4 * (g.lm2l + 1.0) ** -2
    f = {k: (rng.standard_normal((g.lm_max, n_levels)) +
             1j * rng.standard_normal((g.lm_max, n_levels))) * amp[:, None] for k in FIELDS}
    from oracle import stage as ostage

    prof = ostage.bouss_profiles(n_levels, l_max=L_MAX)
    ofast.nl_bouss_stage(g, f, prof, LF, CF, AF, OPM)  # warm
    reps, t = 0, 0.0
    while t < 10.0 and reps < 20:
        t0 = time.perf_counter()
        ofast.nl_bouss_stage(g, f, prof, LF, CF, AF, OPM)
        t += time.perf_counter() - t0
        reps += 1
    per_sample = t / reps
    # synthesis scales with all levels, analysis with bulk levels: scale by levels
    per_step = per_sample * (N_R / n_levels)
    return {"value": 1.0 / per_step, "unit": "steps/s", "cores": os.cpu_count(),
            "threads": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())),
            "kind": "port",
            "sample": f"l_max=255 stage on {n_levels} of {N_R} levels x{reps}, "
                      f"{per_sample:.2f} s each, scaled by {N_R}/{n_levels}; "
                      f"table build {build_s:.1f} s excluded"}


def max_over_ranks(x, dist, device):
    """The largest per-rank value (a step time) over all ranks; x itself with one rank."""
    if dist is None:
        return x
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def job_steps_per_s(world, ms_max):
    """Whole-job throughput of `world` replicas whose slowest one needs ms_max per step."""
    return world * 1000.0 / ms_max


def count_launches(fn):
    """(this library's kernels, all kernels) launched by one call of fn, from the
    CUDA activity of a torch profiler trace (library kernels live in namespace mt)."""
    from torch.profiler import ProfilerActivity, profile

    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    names = [e.name for e in prof.events() if e.device_type.name == "CUDA"
             and not e.name.lower().startswith(("memcpy", "memset"))]
    return sum(1 for n in names if "mt::" in n), len(names)


def run_anel(args, rank, world):
    """Optional line: whole CNAB2 steps of anelastic convection at the anelastic
    benchmark resolution (l_max = 383, n_theta = 576, n_phi = 1152, 129 Chebyshev
    levels, standard (w, p) form; polytropic background with 5 density scale
    heights and index 2, Ek 1e-4, Ra 3e6, Pr 1, no magnetic field, stress-free
    boundaries with the angular-momentum corrections, dt 1e-6; seeded
    perturbations |c_lm| ~ 1e-3 (l+1)^-2), through magic_b200.step.AnelasticStep
    with the stage of --precision (default the fused digit-split stage), beside
    the other two (unless --no-alt): the fused split-precision stage and the
    FP64 stage (composed from the FP64 transform kernels as the reference
    composes it), all with the same FP64 solves; device-timed with the state resident (2.9 GB of spectral
    arrays, larger than L2)."""
    from magic_b200.step import AnelasticStep

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    l_max, n_r = 383, args.levels if args.levels != N_R else 129
    cache = {}

    def build(prec):
        st = AnelasticStep(l_max, n_r, ek=1e-4, ra=3e6, pr=1.0, dt=1e-6, precision=prec,
                           device=dev, cache=cache)
        st.init_random(seed=rank, amp=1e-3)
        for _ in range(args.warmup):
            st.step()
        torch.cuda.synchronize()
        return st

    def timed(st, nsteps, clocks=None):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(nsteps):
            st.step()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / nsteps

    main = args.precision
    st = build(main)
    with ClockSampler(dev) as clocks:
        ms = timed(st, args.steps)
    ours, every = count_launches(lambda: st.step())
    del st
    torch.cuda.empty_cache()
    what = {"split": "the fused split-precision stage (bf16x3 tcgen05 GEMMs, FP32 phi stage)",
            "ozaki": "the fused digit-split stage (int8 digit-plane GEMMs, FP64 phi stage; "
                     "~1e-12 of scale)",
            "fp64": "the FP64 stage (composed from the FP64 transform kernels)"}
    alts = {}
    for prec in ([] if args.no_alt else [q for q in ("fp64", "split", "ozaki") if q != main]):
        sta = build(prec)
        na = max(1, min(args.steps, 3 if prec == "fp64" else 5))
        msa = timed(sta, na)
        alts[prec] = {"value": 1000.0 / msa, "unit": "steps/s", "ms_per_step": msa, "steps": na,
                      "what": "the same steps with " + what[prec]}
        del sta
        torch.cuda.empty_cache()
    if "fp64" in alts:
        alts["fp64"]["speedup"] = alts["fp64"]["ms_per_step"] / ms
    dtype = {"split": "bf16x3/f32 stage, f64 solves", "ozaki": "int8 digits/f64 stage, f64 solves",
             "fp64": "f64"}[main]
    if rank == 0:
        print(json.dumps({"metric": "anelastic CNAB2 steps/s @lmax=383 vs FP64 stage, 1 B200",
                          "value": 1000.0 / ms, "unit": "steps/s", "n_gpus": 1,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": dtype, "data": "synthetic",
                          "config": {"workload": "anelastic convection, whole CNAB2 step "
                                                 "(Chebyshev, standard (w, p) form, "
                                                 "stress-free + AM corrections), " + what[main],
                                     "stage": main,
                                     "l_max": l_max, "n_theta": 576, "n_phi": 1152,
                                     "n_r": n_r, "strat": 5.0, "polind": 2.0, "ek": 1e-4,
                                     "ra": 3e6, "pr": 1.0, "dt": 1e-6, "l_mag": False,
                                     "l2": "state larger than L2", "parallelism": "replicas"},
                          "gpu_launches": ours * args.steps,
                          "kernels_per_step": {"library": ours, "all": every},
                          **{f"{k}_stage": v for k, v in alts.items()},
                          "clocks": clocks.summary()}), flush=True)


def run_td(args, rank, world):
    """Optional line: the explicit time-derivative terms of one step (get_td with the
    double-curl poloidal form + finish_exp radial derivatives, FP64) at l_max = 255 on
    the 97-level fourth-order finite-difference grid, MHD, device-timed with inputs
    resident; roofline against HBM (every input array read once, every output written
    once)."""
    from magic_b200 import Plan
    from magic_b200.profiles import boussinesq_profiles
    from magic_b200.radial import RadialScheme

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n_r = args.levels
    plan = Plan(L_MAX, 1, device=dev)
    sch = RadialScheme(n_r, "FD", fd_order=4, fd_order_bound=2, device=dev)
    g = torch.Generator(device="cpu").manual_seed(rank)
    ins_names = ("Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt", "VxBp",
                 "w", "dw", "ddw", "z", "dz")
    ins = {k: torch.randn(plan.lm_max, n_r, dtype=torch.complex128, generator=g).to(dev)
           for k in ins_names}
    bp = boussinesq_profiles(n_r, L_MAX, device=dev)
    r = torch.as_tensor(sch.r, device=dev)
    prof = dict(r=r, or1=1.0 / r, or2=1.0 / r ** 2, or4=1.0 / r ** 4, orho1=bp["orho1"],
                beta=torch.zeros(n_r, dtype=torch.float64, device=dev))
    out = None

    def step():
        nonlocal out
        out = plan.get_td(ins, prof, 1e5, sch.D1, l_double_curl=True, l_heat=True, l_mag=True,
                          out=out)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clocks:
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    arrays = len(ins_names) + len(out)
    byts = arrays * plan.lm_max * n_r * 16
    peaks, src = measured_peaks()
    ach = byts / (ms * 1e-3) / 1e9
    line = {"metric": "explicit-term assemblies/s (get_td + finish_exp) @lmax=255, 1 B200",
            "value": 1000.0 / ms, "unit": "calls/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "get_td double-curl + finish_exp, MHD, FD4 radial scheme",
                       "l_max": L_MAX, "n_r": n_r, "arrays_in": len(ins_names),
                       "arrays_out": len(out), "l2": "inputs larger than L2"},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": ach / peaks["hbm_gbs"], "traffic": None,
                         "algorithmic_bytes": byts, "peak_source": src},
            "gpu_launches": args.steps, "clocks": clocks.summary()}
    if rank == 0 and not args.no_cpu:
        import numpy as np

        from oracle import td as otd

        sub = 3  # orders m < 3 of the same levels: a bounded CPU sample
        rows = int(np.sum(plan.lm2m < sub))
        h = {k: v[:rows].cpu().numpy() for k, v in ins.items()}
        gg = dict(lm2l=plan.lm2l[:rows], lm2m=plan.lm2m[:rows], l_max=L_MAX, CorFac=1e5,
                  l_anel=0, l_double_curl=1, **{k: v.cpu().numpy() for k, v in prof.items()})
        t0, reps = time.perf_counter(), 0
        while time.perf_counter() - t0 < 3.0:
            otd.get_td(gg, h, sch.D1m)
            reps += 1
        dt = (time.perf_counter() - t0) / reps
        line["cpu_baseline"] = {"value": rows / plan.lm_max / dt, "unit": "calls/s", "cores": 1,
                                "kind": "port",
                                "sample": f"numpy oracle on the {rows} lm rows with m < {sub} "
                                          f"({reps} repeats, 3 s), scaled to all lm_max rows"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def fp64_plain_stage(args, dev, fields, prof, stream, dist):
    """The same stage on an FP64 plan (the plain mode: FP64 DMMA Legendre
    contractions and FP64 phi stage) with the same inputs, device-timed over the
    same number of steps after the same warm-up; ms per stage, max over ranks."""
    from magic_b200 import Plan

    n_r = args.levels
    plan = Plan(L_MAX, 1, precision="fp64", device=dev)
    out = {k: torch.zeros(plan.lm_max, n_r, dtype=torch.complex128, device=dev) for k in OUTS}
    work = torch.zeros(plan.nl_bouss_workspace(n_r, True, False), dtype=torch.uint8, device=dev)
    step = lambda: plan.nl_bouss(fields, prof, LF, CF, AF, OPM, l_mag=True, l_chem=False,
                                 out=out, work=work)
    for _ in range(args.warmup):
        step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)
    del plan, out, work
    torch.cuda.empty_cache()
    return ms


STEP_KERNELS_PER_STEP = 12  # stage: 2 packs + 2 GEMMs + phi + Courant finish; get_td; 5 updates


def cpu_step_sample(n_levels=5, seed=0, budget_s=20.0):
    """A bounded CPU sample of one whole CNAB2 step of the same workload (l_max 255,
    97 FD4 levels, MHD, double curl): the reference's stage algorithm (padded per-m
    matrices, batched matmuls per hemisphere, pocketfft, numpy products) on
    ``n_levels`` levels scaled to all, the explicit terms (get_td) on the rows with
    m < 8 scaled to all rows, and the lm loop as the reference runs it per step: for
    S, Z, W, B, J the CNAB2 right-hand side, pre-factored banded LU solves per degree
    (LAPACK dgbtrs, bands of the FD4 operators: 2 + 2, 4 + 4 for W) and the radial
    derivatives.  Seconds per step."""
    import numpy as np
    import scipy.linalg.lapack as la

    from oracle import fast as ofast
    from oracle import stage as ostage
    from oracle import td as otd

    t0 = time.perf_counter()
    g = ofast.FastGrid(L_MAX)
    build_s = time.perf_counter() - t0
    rng = np.random.default_rng(seed)
    amp = 1e-4 * (g.lm2l + 1.0) ** -2
    cplx = lambda shape: rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    f = {k: cplx((g.lm_max, n_levels)) * amp[:, None] for k in FIELDS}
    prof = ostage.bouss_profiles(n_levels, l_max=L_MAX)

    def timed(fn, budget):
        fn()  # warm
        reps, t = 0, 0.0
        while reps < 1 or (t < budget and reps < 5):
            a = time.perf_counter()
            fn()
            t += time.perf_counter() - a
            reps += 1
        return t / reps, reps

    stage_s, stage_reps = timed(lambda: ofast.nl_bouss_stage(g, f, prof, LF, CF, AF, OPM),
                                budget_s / 2)
    stage_s *= N_R / n_levels
    # explicit terms on the rows with m < msub
    msub = 8
    rows = int(np.sum(g.lm2m < msub))
    from magic_b200.radial import fd_grid, fd_matrices

    r = fd_grid(N_R)
    D1, D2 = fd_matrices(r, 4, 2)[:2]
    ins = {k: cplx((rows, N_R)) for k in ("Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt",
                                          "VxBp", "w", "dw", "ddw", "z", "dz")}
    gg = dict(lm2l=g.lm2l[:rows], lm2m=g.lm2m[:rows], l_max=L_MAX, CorFac=1e5, l_anel=0,
              l_double_curl=1, r=r, or1=1.0 / r, or2=1.0 / r ** 2, or4=1.0 / r ** 4,
              orho1=np.ones(N_R), beta=np.zeros(N_R))
    td_s, _ = timed(lambda: otd.get_td(gg, ins, D1), budget_s / 8)
    td_s *= g.lm_max / rows
    # lm loop: five fields, per-degree banded LU solves with factors built once
    old, impl, e0, e1 = (cplx((g.lm_max, N_R)) for _ in range(4))
    rows_of_l = [np.nonzero(g.lm2l == l)[0] for l in range(L_MAX + 1)]

    def factors(kl):
        out = []
        for l in range(L_MAX + 1):
            ab = np.zeros((2 * kl + kl + 1, N_R))
            ab[kl:2 * kl + 1 + kl] = rng.standard_normal((2 * kl + 1, N_R))
            ab[2 * kl] += 4.0 * kl + 4.0  # diagonal row of the band: diagonally dominant
            lu, piv, _ = la.dgbtrf(ab, kl, kl)
            out.append((lu, piv))
        return out

    fac = {2: factors(2), 4: factors(4)}

    def lm_loop():
        for kl, nder in ((2, 2), (2, 2), (4, 4), (2, 2), (2, 2)):  # S, Z, W (+ p0), B, J
            rhs = old + 0.6 * impl + 1.5 * e0 - 0.5 * e1
            x = np.empty_like(rhs)
            for l in range(L_MAX + 1):
                rr = rows_of_l[l]
                b = np.concatenate([rhs[rr].real, rhs[rr].imag]).T
                lu, piv = fac[kl][l]
                y, _ = la.dgbtrs(lu, kl, kl, np.ascontiguousarray(b), piv)
                x[rr] = y[:, :len(rr)].T + 1j * y[:, len(rr):].T
            d = x
            for k in range(nder):  # dx, d2x (and dddw, ddddw for W)
                d = (d @ (D1 if k % 2 == 0 else D2).T) if k < 2 else (x @ D2.T) @ D1.T
            _ = 0.6 * x + d

    lm_s, lm_reps = timed(lm_loop, budget_s / 4)
    per_step = stage_s + td_s + lm_s
    threads = torch.get_num_threads()
    return {"value": 1.0 / per_step, "unit": "steps/s", "cores": os.cpu_count(),
            "threads": threads, "kind": "port",
            "sample": f"one l_max=255 / 97-level FD4 step: stage on {n_levels} of {N_R} levels "
                      f"x{stage_reps} scaled by {N_R}/{n_levels} ({stage_s:.2f} s), get_td on "
                      f"the {rows} rows with m < {msub} scaled to {g.lm_max} ({td_s:.2f} s), "
                      f"lm loop of 5 fields with pre-factored banded LU x{lm_reps} "
                      f"({lm_s:.2f} s); table build {build_s:.1f} s excluded",
            "s_per_step": per_step}


def step_workload_config(args, prec):
    return {"workload": "Boussinesq MHD dynamo, whole CNAB2 step (" + (
                "FD4 double curl" if args.step_scheme == "FD" else
                "Chebyshev, standard (w, p) form") + f", {prec} stage, FP64 solves)",
            "l_max": args.step_lmax, "minc": 1, "n_r": args.levels, "ek": 1e-5, "ra": 3e8,
            "pr": 1.0, "pm": 1.0, "dt": 2e-7,
            "l2": "state larger than L2 (1.7 GB of spectral arrays)", "parallelism": "replicas"}


def run_step(args, rank, world):
    """Headline: whole CNAB2 time steps of the Boussinesq MHD dynamo (the reference's
    one_step: radial loop with the fused nonlinear stage and the explicit terms, then
    the implicit solves of S, Z, W with the l = 0 pressure, B and J) at l_max = 255 on
    the 97-level fourth-order finite-difference grid (SURVEY config 3: Ek 1e-5, Ra 3e8,
    Pr = Pm = 1, dt 2e-7 fixed, seeded perturbations of amplitude 1e-4 (l+1)^-2),
    device-timed with the state resident; beside it the same steps with the FP64
    stage (the plain FP64 path), per-part times, the dominant kernel's roofline, an
    end-to-end leg through the public step API and a CPU sample.
    --step-lmax / --levels / --step-scheme chebyshev time other shells."""
    from magic_b200.step import BoussinesqStep

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed_steps(st, nsteps, clocks=None):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(nsteps):
            st.step()
        e1.record()
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / nsteps, dist, dev)

    def build(prec):
        st = BoussinesqStep(args.step_lmax, args.levels, ek=1e-5, ra=3e8, pr=1.0, prmag=1.0,
                            dt=2e-7, precision=prec, device=dev, radial_scheme=args.step_scheme)
        st.init_random(seed=rank, amp=1e-4)
        for _ in range(args.warmup):
            st.step()
        torch.cuda.synchronize()
        return st

    def part_times(st):
        """Per-part device times of the same work: synthesis / phi / analysis of the
        stage (the parts mask of the fused stage), get_td, and the lm loop."""
        f = st.f
        fields = {k: f[k] for k in FIELDS}
        stream = torch.cuda.current_stream(dev)
        names = {1: "legendre_synthesis", 2: "phi_fft_products", 4: "legendre_analysis"}
        acc = {v: 0.0 for v in names.values()}
        acc.update(radial_loop=0.0, implicit=0.0)
        # all iterations enqueued back to back and read after one synchronisation,
        # so that the device never idles between an event and the work it
        # brackets (the first iteration, which starts from an idle device, is
        # not counted)
        rounds = []
        for _ in range(args.steps + 1):
            ev = []
            for p in names:
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                st.plan.nl_bouss(fields, st.prof, st.LFfac, 2.5, 1.0, st.opm, l_mag=True,
                                 out=st.nl_out, work=st.work, parts=p)
                b.record(stream)
                ev.append((names[p], a, b))
            a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a.record(stream)
            st.radial_loop()
            b.record(stream)
            st.lm_loop()
            c.record(stream)
            rounds.append((ev, a, b, c))
        torch.cuda.synchronize()
        for ev, a, b, c in rounds[1:]:
            for n, x, y in ev:
                acc[n] += x.elapsed_time(y)
            acc["radial_loop"] += a.elapsed_time(b)
            acc["implicit"] += b.elapsed_time(c)
        out = {k: v / args.steps for k, v in acc.items()}
        out["get_td"] = max(0.0, out["radial_loop"] - sum(out[v] for v in names.values()))
        return out

    prec = args.precision
    st = build(prec)
    with ClockSampler(dev) as clocks:
        ms = timed_steps(st, args.steps)
    value = job_steps_per_s(world, ms)
    parts = part_times(st)
    st.plan.poll_status(block=True)

    # --- end to end through the public step API: the initial state (fields and
    # time arrays) copied in from pinned host memory, then every step's energies
    # (the run's output metric) and Courant limits read back to the host, and the
    # final state copied out; state bytes are counted once per run and divided by
    # the steps.
    k_e2e = max(10, args.steps)
    state = [st.f[k] for k in st.f] + [st.ta[e][k] for e in st.ta for k in st.ta[e]]
    host = [x.cpu().pin_memory() for x in state]
    host_back = [torch.empty(x.shape, dtype=x.dtype).pin_memory() for x in state]
    per_step_out = torch.empty(k_e2e, 2 + 2, dtype=torch.float64)
    lim = torch.empty(2, dtype=torch.float64).pin_memory()
    state_bytes = sum(x.numel() * x.element_size() for x in state)
    st.energies()  # build the energy integrals outside the timed region
    barrier()
    torch.cuda.synchronize()
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea.record()
    for x, h in zip(state, host):
        x.copy_(h, non_blocking=True)
    for i in range(k_e2e):
        dtr, dth = st.step()
        lim.copy_(torch.stack([dtr.min(), dth.min()]), non_blocking=True)
        ek, em = st.energies()  # reads back to the host (synchronises, like .item())
        per_step_out[i] = torch.tensor([ek.e_p + ek.e_t, em.e_p + em.e_t, lim[0], lim[1]],
                                       dtype=torch.float64)
    for x, h in zip(state, host_back):
        h.copy_(x, non_blocking=True)
    eb.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(ea.elapsed_time(eb) / k_e2e, dist, dev)
    assert bool(torch.isfinite(per_step_out).all()), "non-finite energies in the e2e leg"
    st.plan.poll_status(block=True)

    # --- roofline of the dominant kernel of the step
    peaks, src = measured_peaks()
    plan = st.plan
    n_r = args.levels
    kern = {k: parts[k] for k in ("legendre_synthesis", "phi_fft_products",
                                  "legendre_analysis", "get_td")}
    dom = max(kern, key=kern.get)
    split = prec == "split"
    roof = None
    if dom == "phi_fft_products":
        row = plan.n_theta_max * plan.n_m_max * (8 if split else 16)
        byts = (13 * n_r + 9 * (n_r - 2)) * row
        ach = byts / (parts[dom] * 1e-3) / 1e9
        per_row = NCU_PHI_TRAFFIC.get(prec)
        traffic = per_row * (13 * n_r + 9 * (n_r - 2)) if per_row else None
        roof = {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": ach / peaks["hbm_gbs"], "traffic": traffic, "algorithmic_bytes": byts,
                "kernel": dom, "peak_source": src,
                "traffic_source": "ncu dram bytes at n_r=17 scaled by rows" if per_row else None}
        inst_row = NCU_PHI_INST.get(prec)
        if inst_row:
            props = torch.cuda.get_device_properties(dev)
            mhz = clocks.summary().get("sm_mhz") or 1965.0
            inst = inst_row * (13 * n_r + 9 * (n_r - 2))
            rate = inst / (parts[dom] * 1e-3)
            peak_issue = props.multi_processor_count * 4 * mhz * 1e6
            roof["issue"] = {"warp_instructions": inst, "achieved": rate, "peak": peak_issue,
                             "unit": "warp inst/s", "frac": rate / peak_issue,
                             "source": "ncu smsp__inst_executed.sum at n_r=17 scaled by rows"}
    elif dom == "get_td":
        byts = 18 * plan.lm_max * n_r * 16
        ach = byts / (parts[dom] * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": ach / peaks["hbm_gbs"], "traffic": None, "algorithmic_bytes": byts,
                "kernel": dom, "peak_source": src}
    elif split:
        s_mma, a_mma = split_mma_flops(plan, n_r)
        fl = s_mma if dom == "legendre_synthesis" else a_mma
        pk = peaks["bf16_tflops"]
        ach = fl / (parts[dom] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": ach / pk, "traffic": None, "kernel": dom,
                "flops": "dense bf16 MMA FLOPs issued (6 plane products, padded tiles)",
                "peak_source": f"{src} bf16_tflops (burst)"}
    elif prec == "ozaki":
        s_mma, a_mma = ozaki_mma_ops(plan, n_r)
        fl = s_mma if dom == "legendre_synthesis" else a_mma
        pk = 2.0 * peaks["bf16_tflops"]
        ach = fl / (parts[dom] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": pk, "unit": "TOP/s",
                "frac": ach / pk, "traffic": None, "kernel": dom,
                "flops": "dense int8 MMA operations issued (21 digit pairs per K chunk in "
                         "eight stacked MMAs, padded tiles; the pack kernel's time is included "
                         "in the part)",
                "peak_source": f"2 x {src} bf16_tflops (burst): B200's dense int8 rate is "
                               "twice its bf16 rate"}
    else:
        synth_f, anal_f = flops_per_step(plan.nhs, plan.lm_max, n_r)
        fl = synth_f if dom == "legendre_synthesis" else anal_f
        pk = dgemm_peak(dev) if rank == 0 else float("nan")
        ach = fl / (parts[dom] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": ach / pk, "traffic": None, "kernel": dom,
                "peak_source": "cuBLAS FP64 DGEMM 8192^3 measured in this run "
                               "(no FP64 entry in MEASURED_PEAKS.json)"}
    synth_f, anal_f = flops_per_step(plan.nhs, plan.lm_max, n_r)
    sht_tflops = (synth_f + anal_f) / ((parts["legendre_synthesis"] +
                                        parts["legendre_analysis"]) * 1e-3) / 1e12
    del st, state, host, host_back
    torch.cuda.empty_cache()

    # --- the plain FP64 path: the same steps with the FP64 stage; and the
    # bf16x3 / FP32 split stage (fastest, ~1e-6 of scale per stage)
    plain = None
    other = {}
    if prec != "fp64":
        sf = build("fp64")
        plain_ms = timed_steps(sf, args.steps)
        plain = {"value": job_steps_per_s(world, plain_ms), "unit": "steps/s",
                 "ms_per_step": plain_ms, "speedup": plain_ms / ms,
                 "what": "the same whole steps with the FP64 stage (DMMA Legendre, FP64 phi "
                         "stage) and the same FP64 solves, device-timed",
                 "kernel_ms": part_times(sf)}
        del sf
        torch.cuda.empty_cache()
    for alt in ("split",):
        if alt == prec or args.no_alt:
            continue
        sa = build(alt)
        alt_ms = timed_steps(sa, args.steps)
        other[alt] = {"value": job_steps_per_s(world, alt_ms), "unit": "steps/s",
                      "ms_per_step": alt_ms,
                      "what": "the same whole steps with the bf16x3 / FP32-accumulate split "
                              "stage and FP32 phi stage (~1e-6 of scale per stage)",
                      "kernel_ms": part_times(sa)}
        del sa
        torch.cuda.empty_cache()
    drift = measure_drift(args, dev, rank) if args.drift_steps > 0 else None

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": {"split": "bf16x3/f32 stage, f64 solves",
                          "ozaki": "int8 digit planes (exact int32 accumulation, f64 combine), "
                                   "f64 phi stage and solves"}.get(prec, "f64"),
                "data": "synthetic", "config": step_workload_config(args, prec),
                "clocks": clocks.summary(),
                "e2e": {"value": job_steps_per_s(world, e2e_ms), "unit": "steps/s",
                        "h2d_bytes_per_step": state_bytes / k_e2e,
                        "d2h_bytes_per_step": state_bytes / k_e2e + 32,
                        "ms_per_step": e2e_ms, "steps": k_e2e,
                        "what": "initial state in from pinned host memory, steps through "
                                "BoussinesqStep.step with every step's energies and Courant "
                                "limits read back, final state out"},
                "gpu_launches": STEP_KERNELS_PER_STEP * args.steps,
                "kernel_ms": parts, "sht_tflops": sht_tflops, "roofline": roof}
        if plain is not None:
            line["fp64_plain"] = plain
        for k, v in other.items():
            line[f"{k}_stage"] = v
        if drift:
            line["drift"] = drift
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_step_sample()
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_serve(args, rank, world):
    """Optional line: the ensemble stream (Poisson arrivals at 4 runs/s, l_max in
    {32, 64, 85, 127}, n_r in {33, 49, 65}, Ek log-uniform [1e-4, 1e-3], Ra
    log-uniform [1e5, 1e6], Pr 1, Pm 5, perturbation 1e-5, Boussinesq MHD steps on
    Chebyshev levels (standard (w, p) form) at dt 1e-4) served with continuous batching in split
    precision: p50 / p99 per-step device latency and aggregate steps/s over the
    serving wall time (value).  The same runs all arriving at once measure the
    capacity.  Baseline: the FP64 stage one run at a time, eager: each run's
    build time (host clock) and steps (device events) measured, then replayed
    against the same arrival times (run i starts when it has arrived and run
    i - 1 is done) for its stream wall time, and summed for its capacity."""
    import dataclasses

    from magic_b200.serve import EnsembleServer, latency_report, poisson_stream
    from magic_b200.step import BoussinesqStep

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from magic_b200.serve import BatchedEnsembleServer

    specs = poisson_stream(args.serve_runs, rate=4.0, seed=rank, n_steps=args.serve_steps)
    srv = EnsembleServer(device=dev)
    with ClockSampler(dev) as clocks:
        rep = latency_report(srv.serve(specs), srv.wall_s)
    sat_specs = [dataclasses.replace(s, arrival=0.0) for s in specs]
    srv = EnsembleServer(device=dev)
    sat = latency_report(srv.serve(sat_specs), srv.wall_s)
    # cross-run batching: one fused stage per resolution group per step, in the
    # split mode and in the digit-split mode that meets the precision bounds
    batched = {}
    for prec in ("split", "ozaki"):
        for name, ss in (("stream", specs), ("capacity", sat_specs)):
            bsrv = BatchedEnsembleServer(device=dev)
            res = bsrv.serve([dataclasses.replace(s, precision=prec) for s in ss])
            r = latency_report(res, bsrv.wall_s)
            r["kernels_per_run_step"] = (sum(g.kernel_launches for g in bsrv.groups.values()) /
                                         max(1, r["steps"]))
            r["group_steps"] = sum(g.launches for g in bsrv.groups.values())
            batched[f"{prec}_{name}"] = r
        torch.cuda.empty_cache()
    finish, busy, steps_s, step_ms = 0.0, 0.0, 0.0, []
    for s in specs:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = BoussinesqStep(s.l_max, s.n_r, ek=s.ek, ra=s.ra, pr=s.pr, prmag=s.prmag, dt=s.dt,
                            precision="fp64", device=dev, radial_scheme=s.radial_scheme)
        st.init_random(seed=s.seed, amp=s.amp)
        torch.cuda.synchronize()
        build = time.perf_counter() - t0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(s.n_steps):
            st.step()
        e1.record()
        torch.cuda.synchronize()
        dev_s = e0.elapsed_time(e1) / 1e3
        run_s = build + dev_s
        finish = max(finish, s.arrival) + run_s
        busy += run_s
        steps_s += dev_s
        step_ms.append(1e3 * dev_s / s.n_steps)
        del st
    torch.cuda.empty_cache()
    # accuracy of the serving precisions over whole runs: one spec of each l_max
    # of the stream (its Ek, Ra, n_r, seed), all steps, against the same run with
    # the FP64 stage: largest field difference over the largest field value, and
    # the largest relative difference of the kinetic and magnetic energies
    accuracy = {}
    seen = {}
    for s in specs:
        seen.setdefault(s.l_max, s)
    for l_max, s in sorted(seen.items()):
        runs = {}
        for prec in ("fp64", "split", "ozaki"):
            st = BoussinesqStep(s.l_max, s.n_r, ek=s.ek, ra=s.ra, pr=s.pr, prmag=s.prmag,
                                dt=s.dt, precision=prec, device=dev,
                                radial_scheme=s.radial_scheme)
            st.init_random(seed=s.seed, amp=s.amp)
            for _ in range(s.n_steps):
                st.step()
            torch.cuda.synchronize()
            ek, em = st.energies()
            runs[prec] = ({k: st.f[k].clone() for k in ("w", "z", "s", "b", "aj")},
                          [ek[0], ek[1], em[0], em[1]])
            del st
        ref_f, ref_e = runs["fp64"]
        for prec in ("split", "ozaki"):
            f, e = runs[prec]
            fe = max(float((f[k] - ref_f[k]).abs().max() / ref_f[k].abs().max()) for k in f)
            ee = max(abs(x - y) / abs(y) for x, y in zip(e, ref_e) if y != 0.0)
            accuracy[f"{prec}_l{l_max}_n{s.n_r}"] = {"fields": fe, "energies": ee,
                                                     "steps": s.n_steps}
        torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps({
            "metric": "ensemble aggregate steps/s (continuous batching), 1 B200",
            "value": rep["steps_per_s"], "unit": "steps/s", "n_gpus": 1,
            "higher_is_better": True, "p50_ms": rep["p50_ms"], "p99_ms": rep["p99_ms"],
            "runs": rep["runs"], "steps": rep["steps"], "wall_s": rep["wall_s"],
            "last_arrival_s": specs[-1].arrival,
            "capacity": {"steps_per_s": sat["steps_per_s"], "p50_ms": sat["p50_ms"],
                         "p99_ms": sat["p99_ms"], "wall_s": sat["wall_s"]},
            "fp64_one_at_a_time": {"steps_per_s": rep["steps"] / finish, "wall_s": finish,
                                   "capacity_steps_per_s": rep["steps"] / busy,
                                   "steps_per_s_without_build": rep["steps"] / steps_s,
                                   "run_mean_step_ms_p50": statistics.median(step_ms),
                                   "run_mean_step_ms_max": max(step_ms)},
            "accuracy_vs_fp64": accuracy,
            "kernels_per_run_step": 12,
            "batched": batched,
            "dtype": "bf16x3/f32 stage, f64 rest", "data": "synthetic",
            "config": {"workload": "ensemble stream: Poisson 4 runs/s, l_max 32-127, n_r 33-65, "
                                   "Chebyshev Boussinesq MHD, dt 1e-4",
                       "runs": args.serve_runs, "steps_per_run": args.serve_steps},
            "clocks": clocks.summary()}), flush=True)


def run_sht(args, rank, world):
    """Optional line: the standalone SHT round trip (l_max = 127, n_theta = 192,
    n_phi = 384, minc = 1) batched over 65 radial levels x (1 scalar + 2 torpol
    vector fields) through the drop-in transforms: scal_to_spat -> scal_to_SH on
    the 65 scalar columns; torpol_to_spat -> scal_to_SH (br) + spat_to_sphertor
    (bt, bp) on the 130 vector columns.  |c_lm| = (l+1)^-2 with phases uniform
    from seed 0 (m = 0 real).  Per mode (FP64 and split): device time per round
    trip, SHT TFLOP/s with the flop convention F = 4 n_theta/2 lm_max per
    scalar-equivalent contraction and column (18 F per level: 1 + 1 scalar,
    2 x (3 + 1 + 4) vector), and the round trip's relative error against its
    input (largest value of each array; S, T from l >= 1)."""
    from magic_b200 import Plan

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L_SHT, LEV = 127, 65
    res = {}
    for prec in ("split", "fp64"):
        plan = Plan(L_SHT, 1, precision=prec, device=dev)
        l = torch.as_tensor(plan.lm2l, dtype=torch.float64)
        m0 = torch.as_tensor(plan.lm2m == 0)
        g = torch.Generator(device="cpu").manual_seed(0)

        def spec(B):
            ph = torch.rand(plan.lm_max, B, generator=g, dtype=torch.float64) * 2 * math.pi
            c = torch.polar(((l + 1.0) ** -2)[:, None].expand(-1, B).contiguous(), ph)
            c[m0] = c[m0].real.to(c.dtype)
            return c.to(dev)

        sc, Q, S, T = spec(LEV), spec(2 * LEV), spec(2 * LEV), spec(2 * LEV)

        def round_trip():
            sc2 = plan.scal_to_SH(plan.scal_to_spat(sc))
            br, bt, bp = plan.torpol_to_spat(Q, S, T)
            return sc2, plan.scal_to_SH(br), *plan.spat_to_sphertor(bt, bp)

        for _ in range(args.warmup):
            round_trip()
        torch.cuda.synchronize()
        # the round trip (five transform calls, ~0.5 ms of device work) captured
        # once as a CUDA graph and replayed, so that the host's launch rate (and
        # the clock sampler's driver calls beside it) do not pace the device
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            round_trip()
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize()
        with torch.cuda.graph(graph):
            out = round_trip()
        graph.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev) as clocks:
            e0.record()
            for _ in range(args.steps):
                graph.replay()
            e1.record()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        plan.poll_status(block=True)
        lpos = (l > 0).to(dev)
        rel = lambda a, b: float((a - b).abs().max() / b.abs().max())
        errs = {"scalar": rel(out[0], sc), "Q": rel(out[1], Q),
                "S": rel(out[2][lpos], S[lpos]), "T": rel(out[3][lpos], T[lpos])}
        flops = LEV * 18 * 4.0 * plan.nhs * plan.lm_max
        res[prec] = dict(ms=ms, tflops=flops / (ms * 1e-3) / 1e12, round_trip_rel_err=errs,
                         clocks=clocks.summary())
        del graph, out
        del plan
        torch.cuda.empty_cache()
    if rank == 0:
        sp, fp = res["split"], res["fp64"]
        peaks, src = measured_peaks()
        print(json.dumps({
            "metric": "SHT round-trip TFLOP/s @lmax=127, 65 levels x (1 scalar + 2 torpol), 1 B200",
            "value": sp["tflops"], "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sp["ms"], "higher_is_better": True,
            "dtype": "bf16x3/f32", "data": "synthetic",
            "config": {"workload": "SHT round trip through the drop-in transforms", "l_max": L_SHT,
                       "n_theta": 192, "n_phi": 384, "levels": LEV,
                       "columns": {"scalar": LEV, "torpol": 2 * LEV},
                       "flops_per_round_trip": LEV * 18 * 4.0 * 96 * 8256,
                       "l2": "grids 268 MB per round trip, larger than L2"},
            "round_trip_rel_err": sp["round_trip_rel_err"],
            "fp64": {"value": fp["tflops"], "ms_per_step": fp["ms"],
                     "round_trip_rel_err": fp["round_trip_rel_err"]},
            "split_over_fp64": fp["ms"] / sp["ms"],
            "peak_bf16_tflops": peaks["bf16_tflops"], "peak_source": src,
            "clocks": sp["clocks"]}), flush=True)


def measure_drift(args, dev, rank):
    """The split stage's drift from the FP64 stage: both run args.drift_steps whole
    steps from the same seeded state; max over w, z, s, b, aj of |split - fp64| /
    max |fp64| per field, and the largest relative difference of the four total
    energies (kinetic / magnetic, poloidal / toroidal)."""
    from magic_b200.step import BoussinesqStep

    runs = []
    for prec in ("fp64", "split"):
        st = BoussinesqStep(L_MAX, args.levels, ek=1e-5, ra=3e8, pr=1.0, prmag=1.0, dt=2e-7,
                            precision=prec, device=dev)
        st.init_random(seed=rank, amp=1e-4)
        runs.append(st)
    a, b = runs
    for _ in range(args.drift_steps):
        a.step()
        b.step()
    torch.cuda.synchronize()
    fe = {k: ((a.f[k] - b.f[k]).abs().max() / a.f[k].abs().max()).item()
          for k in ("w", "z", "s", "b", "aj")}
    ea, eb = a.energies(), b.energies()
    pairs = list(zip(ea[0][:2] + ea[1][:2], eb[0][:2] + eb[1][:2]))
    return {"steps": args.drift_steps, "field_rel": fe, "field_rel_max": max(fe.values()),
            "energy_rel_max": max(abs(x - y) / abs(x) for x, y in pairs),
            "energies_fp64": {"e_kin_pol": ea[0][0], "e_kin_tor": ea[0][1],
                              "e_mag_pol": ea[1][0], "e_mag_tor": ea[1][1]}}


def run_reference(args, rank, world):
    """The reference arm: the reference's CPU algorithm for the same whole step
    (cpu_step_sample: a port, the reference itself does not travel), timed on this
    host's cores with all threads torch offers; one warm-up sample and up to
    min(steps, 3) timed samples (each is one whole step of the workload, assembled
    from bounded parts as cpu_step_sample says).  Under torchrun only rank 0 runs."""
    if rank != 0:
        return
    n = max(1, min(args.steps, 3))
    cpu_step_sample(budget_s=4.0)  # warm-up sample (imports, tables, allocator)
    samples = [cpu_step_sample(seed=i, budget_s=4.0) for i in range(n)]
    s_per = statistics.median(x["s_per_step"] for x in samples)
    v = 1.0 / s_per
    base = dict(samples[0], value=v)
    line = {"metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": n,
            "warmup": 1, "ms_per_step": 1000.0 * s_per, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": step_workload_config(args, "fp64 CPU port"),
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "steps = whole-step samples actually timed (each the median-free sum of "
                    "its bounded parts); the reference is Python and is not installed here, "
                    "so its algorithm runs as the committed CPU port"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="ozaki", choices=["fp64", "split", "ozaki"],
                    help="stage precision of the timed steps: ozaki (digit-split tensor-core "
                         "Legendre + FP64 phi stage, the mode that meets the precision bounds), "
                         "split (bf16x3 / FP32), fp64")
    ap.add_argument("--no-alt", action="store_true", help="skip the alternative split leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--workload", default="step",
                    choices=["step", "stage", "anel", "td", "serve", "sht"],
                    help="step (headline): whole CNAB2 time steps at l_max=255, 97 FD4 levels, "
                         "beside the plain FP64 path; stage: the Boussinesq MHD nonlinear "
                         "stage alone (extra line); sht: the standalone SHT round trip at "
                         "l_max=127 (extra line); anel: whole anelastic CNAB2 steps at "
                         "l_max=383, 129 Chebyshev levels (extra line, split and FP64 "
                         "stages); td: the explicit "
                         "time-derivative terms (get_td + finish_exp, FP64, extra line); "
                         "serve: the ensemble stream, continuous batching (extra line)")
    ap.add_argument("--step-lmax", type=int, default=L_MAX, help="step: l_max of the shell")
    ap.add_argument("--step-scheme", default="FD", choices=["FD", "chebyshev"],
                    help="step: radial scheme (FD4 double curl or Chebyshev standard form)")
    ap.add_argument("--serve-runs", type=int, default=64, help="serve: runs in the stream")
    ap.add_argument("--serve-steps", type=int, default=200, help="serve: steps per run")
    ap.add_argument("--drift-steps", type=int, default=0,
                    help="step workload: also run both stages this many steps from one seeded "
                         "state and report the split stage's drift from the FP64 one")
    ap.add_argument("--levels", type=int, default=N_R,
                    help="radial levels (profiling runs use fewer than the 97 of the workload)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "anel":
        run_anel(args, rank, world)
        return
    if args.workload == "td":
        run_td(args, rank, world)
        return
    if args.workload == "step":
        run_step(args, rank, world)
        return
    # --workload stage: the nonlinear stage alone
    if args.workload == "serve":
        run_serve(args, rank, world)
        return
    if args.workload == "sht":
        run_sht(args, rank, world)
        return

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    from magic_b200 import Plan
    from magic_b200.profiles import boussinesq_profiles

    n_r = args.levels
    plan = Plan(L_MAX, 1, precision=args.precision, device=dev)
    fields = synth_inputs(plan, n_r, dev, seed=rank)
    prof = boussinesq_profiles(n_r, L_MAX, device=dev)
    out = {k: torch.zeros(plan.lm_max, n_r, dtype=torch.complex128, device=dev) for k in OUTS}
    work = torch.empty(plan.nl_bouss_workspace(n_r, True, False), dtype=torch.uint8, device=dev)

    work.zero_()

    def step(parts=0):
        return plan.nl_bouss(fields, prof, LF, CF, AF, OPM, l_mag=True, l_chem=False, out=out,
                             work=work, parts=parts)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # --- headline: device-timed whole stage, inputs resident in HBM
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)
    value = job_steps_per_s(world, ms)

    # --- per-kernel times: same work, each part bracketed by events on the same stream
    parts = {1: "legendre_synthesis", 2: "phi_fft_products", 4: "legendre_analysis"}
    ev = {p: [] for p in parts}
    for _ in range(args.steps):
        for p in parts:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step(p)
            b.record(stream)
            ev[p].append((a, b))
    torch.cuda.synchronize()
    part_ms = {parts[p]: sum(a.elapsed_time(b) for a, b in ev[p]) / len(ev[p]) for p in parts}

    # --- end to end through the public API with pinned host buffers: every
    # step copies its 11 input spectra host->device and its 8 output spectra and
    # the Courant steps device->host; copies of neighbouring steps overlap the
    # stage on separate streams (NB buffer sets of device inputs and outputs).
    if args.no_e2e:
        if rank == 0:
            print(json.dumps({"levels": n_r, "ms_per_step": ms, "kernel_ms": part_ms}), flush=True)
        return
    host_in = {k: v.cpu().pin_memory() for k, v in fields.items()}
    NB = 3
    dev_in = [{k: torch.empty_like(v) for k, v in fields.items()} for _ in range(NB)]
    dev_out = [{k: torch.zeros_like(v) for k, v in out.items()} for _ in range(NB)]
    host_out = [{k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in out.items()}
                for _ in range(NB)]
    host_dt = [torch.empty(2, n_r, dtype=torch.float64).pin_memory() for _ in range(NB)]
    h2d = sum(v.numel() * v.element_size() for v in host_in.values())
    d2h = sum(v.numel() * v.element_size() for v in host_out[0].values()) + host_dt[0].numel() * 8
    s_in = torch.cuda.Stream(dev)
    s_out = torch.cuda.Stream(dev)
    ev = lambda: torch.cuda.Event()
    used = [ev() for _ in range(NB)]     # stage of buffer b finished (inputs free, outputs ready)
    copied = [ev() for _ in range(NB)]   # inputs of buffer b on the device
    drained = [ev() for _ in range(NB)]  # outputs of buffer b on the host
    for b in range(NB):
        used[b].record(stream)
        drained[b].record(stream)

    def e2e_step(i):
        b = i % NB
        with torch.cuda.stream(s_in):
            s_in.wait_event(used[b])
            for k in FIELDS:
                dev_in[b][k].copy_(host_in[k], non_blocking=True)
            copied[b].record(s_in)
        stream.wait_event(copied[b])
        stream.wait_event(drained[b])
        o, dtr, dth = plan.nl_bouss(dev_in[b], prof, LF, CF, AF, OPM, l_mag=True, out=dev_out[b],
                                    work=work)
        used[b].record(stream)
        with torch.cuda.stream(s_out):
            s_out.wait_event(used[b])
            for k in OUTS:
                host_out[b][k].copy_(o[k], non_blocking=True)
            host_dt[b][0].copy_(dtr, non_blocking=True)
            host_dt[b][1].copy_(dth, non_blocking=True)
            drained[b].record(s_out)

    for i in range(NB):
        e2e_step(i)
    torch.cuda.synchronize()
    k_e2e = max(10, args.steps)
    barrier()
    torch.cuda.synchronize()
    a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a_ev.record(stream)
    for i in range(k_e2e):
        e2e_step(i)
    for b in range(NB):
        stream.wait_event(drained[b])
    b_ev.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(a_ev.elapsed_time(b_ev) / k_e2e, dist, dev)

    # --- roofline of the dominant kernel
    peaks, src = measured_peaks()
    synth_f, anal_f = flops_per_step(plan.nhs, plan.lm_max, n_r)
    dom = max(part_ms, key=part_ms.get)
    roof = None
    split = args.precision == "split"
    if dom == "phi_fft_products":
        # algorithmic bytes: Fourier rows in (13 fields x n_r levels) and out
        # (9 fields x (n_r - 2) levels), each n_theta x n_m complex values
        # (FP64 complex in the plain path; FP32 sym/asym in, FP32 north/south
        # out in the split path)
        row = plan.n_theta_max * plan.n_m_max * (8 if split else 16)
        byts = (13 * n_r + 9 * (n_r - 2)) * row
        ach = byts / (part_ms[dom] * 1e-3) / 1e9
        per_row = NCU_PHI_TRAFFIC.get(args.precision)
        traffic = per_row * (13 * n_r + 9 * (n_r - 2)) if per_row else None
        roof = {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": ach / peaks["hbm_gbs"], "traffic": traffic, "algorithmic_bytes": byts,
                "kernel": dom, "peak_source": src,
                "traffic_source": "ncu dram bytes at n_r=17 scaled by rows" if per_row else None}
        # the kernel is issue-bound, not HBM-bound: warp instructions per second
        # against the SM partitions' issue peak (one warp instruction per clock
        # per partition, 4 partitions per SM) at the clock sampled in the run
        inst_row = NCU_PHI_INST.get(args.precision)
        if inst_row:
            props = torch.cuda.get_device_properties(dev)
            mhz = clocks.summary().get("sm_mhz") or 1965.0
            inst = inst_row * (13 * n_r + 9 * (n_r - 2))
            rate = inst / (part_ms[dom] * 1e-3)
            peak_issue = props.multi_processor_count * 4 * mhz * 1e6
            roof["issue"] = {"warp_instructions": inst, "achieved": rate, "peak": peak_issue,
                             "unit": "warp inst/s", "frac": rate / peak_issue,
                             "source": "ncu smsp__inst_executed.sum at n_r=17 scaled by rows"}
    elif split:
        s_mma, a_mma = split_mma_flops(plan, n_r)
        fl = s_mma if dom == "legendre_synthesis" else a_mma
        pk = peaks["bf16_tflops"]
        ach = fl / (part_ms[dom] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": ach / pk, "traffic": None, "kernel": dom,
                "flops": "dense bf16 MMA FLOPs issued (6 plane products, padded tiles)",
                "peak_source": f"{src} bf16_tflops (burst)"}
    elif args.precision == "ozaki":
        s_mma, a_mma = ozaki_mma_ops(plan, n_r)
        fl = s_mma if dom == "legendre_synthesis" else a_mma
        pk = 2.0 * peaks["bf16_tflops"]
        ach = fl / (part_ms[dom] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": pk, "unit": "TOP/s",
                "frac": ach / pk, "traffic": None, "kernel": dom,
                "flops": "dense int8 MMA operations issued (21 digit pairs per K chunk)",
                "peak_source": f"2 x {src} bf16_tflops (burst)"}
    else:
        fl = synth_f if dom == "legendre_synthesis" else anal_f
        pk = dgemm_peak(dev) if rank == 0 else float("nan")
        ach = fl / (part_ms[dom] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": ach / pk, "traffic": None, "kernel": dom,
                "peak_source": "cuBLAS FP64 DGEMM 8192^3 measured in this run "
                               "(no FP64 entry in MEASURED_PEAKS.json)"}
    sht_tflops = (synth_f + anal_f) / ((part_ms["legendre_synthesis"] +
                                        part_ms["legendre_analysis"]) * 1e-3) / 1e12
    plain = (fp64_plain_stage(args, dev, fields, prof, stream, dist)
             if args.precision != "fp64" else None)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": {"split": "bf16x3/f32", "ozaki": "int8 digits/f64"}.get(
                    args.precision, "f64"), "data": "synthetic",
                "config": workload_config(args.precision),
                "clocks": clocks.summary(),
                "e2e": {"value": job_steps_per_s(world, e2e_ms), "unit": "steps/s",
                        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": e2e_ms},
                "gpu_launches": 6 * args.steps,  # split: 2 packs, 2 GEMMs, phi, Courant; fp64: 2 + 1 + 2 + 1
                "kernel_ms": part_ms, "sht_tflops": sht_tflops,
                "roofline": roof}
        if plain is not None:
            line["fp64_plain"] = {"value": job_steps_per_s(world, plain), "unit": "steps/s",
                                  "ms_per_step": plain, "split_over_fp64": plain / ms,
                                  "what": "the same stage on an FP64 plan (DMMA Legendre, "
                                          "FP64 phi stage), same inputs, device-timed",
                                  "gpu_launches": 6 * args.steps}
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_stage_sample()
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
