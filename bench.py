"""Benchmark: the Boussinesq MHD nonlinear stage at l_max=255 on B200.

One step = one nonlinear stage of the radial loop (magic_torch/step_time.py:
931-1213, transforms + get_nl + Courant): Legendre synthesis of 13 grid fields
on all n_r = 97 levels, the fused phi-FFT + products + Courant kernel, and the
Legendre analysis of the 9 spectral outputs on the 95 bulk levels, at
l_max = 255 (n_theta = 384, n_phi = 768, minc = 1) with magnetic field and no
composition.  Synthetic seeded spectral fields (|c_lm| ~ 1e-4 (l+1)^-2);
random-phase inputs larger than L2 (561 MB of spectral inputs per step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) each rank runs an independent replica of the workload
(the stage has no cross-GPU exchange); value = total steps/s over all ranks.
"""

import argparse
import json
import math
import os
import statistics
import subprocess
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
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        load = sorted(sm)[len(sm) // 2:] if len(sm) > 4 else sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


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


def run_reference(args, rank, world):
    if rank != 0:
        return
    base = cpu_stage_sample()
    steps = max(1, args.steps)
    vals = [cpu_stage_sample(seed=i)["value"] for i in range(1)]
    v = statistics.median(vals + [base["value"]])
    line = {"metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": workload_config("fp64, CPU restatement"),
            "cpu_baseline": dict(base, value=v),
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="split", choices=["fp64", "split"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
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
    with ClockSampler(dev.index) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    if dist is not None:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = t.item()
    value = world * 1000.0 / ms

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

    # --- end to end through the public API with pinned host buffers
    if args.no_e2e:
        if rank == 0:
            print(json.dumps({"levels": n_r, "ms_per_step": ms, "kernel_ms": part_ms}), flush=True)
        return
    host_in = {k: v.cpu().pin_memory() for k, v in fields.items()}
    host_out = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in out.items()}
    host_dt = torch.empty(2, n_r, dtype=torch.float64).pin_memory()
    dev_in = {k: torch.empty_like(v) for k, v in fields.items()}
    h2d = sum(v.numel() * v.element_size() for v in host_in.values())
    d2h = sum(v.numel() * v.element_size() for v in host_out.values()) + host_dt.numel() * 8

    def e2e_step():
        for k in FIELDS:
            dev_in[k].copy_(host_in[k], non_blocking=True)
        o, dtr, dth = plan.nl_bouss(dev_in, prof, LF, CF, AF, OPM, l_mag=True, out=out, work=work)
        for k in OUTS:
            host_out[k].copy_(o[k], non_blocking=True)
        host_dt[0].copy_(dtr, non_blocking=True)
        host_dt[1].copy_(dth, non_blocking=True)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    k_e2e = max(3, args.steps // 2)
    barrier()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(k_e2e):
        e2e_step()
    b.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = a.elapsed_time(b) / k_e2e
    if dist is not None:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = t.item()

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
        roof = {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": ach / peaks["hbm_gbs"], "traffic": None, "kernel": dom,
                "peak_source": src}
    elif split:
        s_mma, a_mma = split_mma_flops(plan, n_r)
        fl = s_mma if dom == "legendre_synthesis" else a_mma
        pk = peaks["bf16_tflops"]
        ach = fl / (part_ms[dom] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": ach / pk, "traffic": None, "kernel": dom,
                "flops": "dense bf16 MMA FLOPs issued (6 plane products, padded tiles)",
                "peak_source": f"{src} bf16_tflops (burst)"}
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

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "bf16x3/f32" if split else "f64", "data": "synthetic",
                "config": workload_config(args.precision),
                "clocks": clocks.summary(),
                "e2e": {"value": world * 1000.0 / e2e_ms, "unit": "steps/s",
                        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": e2e_ms},
                "gpu_launches": (4 if split else 6) * args.steps,
                "kernel_ms": part_ms, "sht_tflops": sht_tflops,
                "roofline": roof}
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_stage_sample()
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
