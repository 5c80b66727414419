"""Ensemble serving loop: independent dynamo runs on one GPU.

Runs (RunSpec: l_max, n_r, Ekman, Rayleigh, ... and an arrival time) come in
as a stream.  The loop admits a run as soon as it has arrived, a slot is free
and its device-memory footprint fits the budget; the run then keeps its
spectral fields and time arrays resident (one BoussinesqStep; transform
plans, radial operators and factored solve operators are resident once per
shape and shared by the runs of that shape) and steps on its own CUDA stream through a CUDA graph
captured after its first step, so the steps of all admitted runs overlap on
the device.  A run that has done its steps reports its energies (and, on
request, its final state in the reference's checkpoint layout), frees its
memory and its slot, and the next waiting run is admitted: continuous
batching, not a queue.  Per-step latency is the device time between events
recorded before and after each step on the run's stream; the report gives
p50 / p99 over all steps beside the aggregate steps/s.

The reference has no serving loop; its unit of work is one run
(magic_torch/main.py:280-850), whose step is reproduced here by
BoussinesqStep.  A step is a graph replay of the same kernels on the same
buffers as an eager step, so a run's result does not depend on which other
runs share the GPU (tests/test_gpu_serve.py checks this bit for bit).
"""

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch


@dataclass
class RunSpec:
    run_id: int
    l_max: int
    n_r: int
    ek: float
    ra: float
    pr: float = 1.0
    prmag: float = 5.0
    dt: float = 1e-4
    n_steps: int = 200
    seed: int = 0
    amp: float = 1e-5
    arrival: float = 0.0  # seconds after the start of serving
    precision: str = "split"
    radial_scheme: str = "chebyshev"  # the reference's default; "FD": fourth-order FD


@dataclass
class RunResult:
    spec: RunSpec
    energies: tuple = None          # (EKin, EMagOC) after the last step
    state: dict = None              # reference checkpoint dictionary (keep_state)
    latencies_ms: list = field(default_factory=list)
    admitted_s: float = 0.0
    finished_s: float = 0.0


def poisson_stream(n_runs=64, rate=4.0, seed=0, n_steps=200, precision="split",
                   l_choices=(32, 64, 85, 127), nr_choices=(33, 49, 65),
                   radial_scheme="chebyshev"):
    """Seeded run stream: exponential inter-arrival times of mean 1 / rate,
    l_max and n_r uniform over the choices, Ekman log-uniform in [1e-4, 1e-3],
    Rayleigh log-uniform in [1e5, 1e6], Pr = 1, Pm = 5, perturbation 1e-5.  The
    time step is the largest of 1e-5, 2e-5, 5e-5, 1e-4 not above Ek / 10: the
    Coriolis term is explicit in the CNAB2 scheme (get_td), so a stable dt
    shrinks with Ek (1e-4 at Ek = 1e-3, as in the reference's shell case), and
    runs of one dt share their solve operators."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_runs):
        t += rng.exponential(1.0 / rate)
        l_max, n_r = int(rng.choice(l_choices)), int(rng.choice(nr_choices))
        ek = float(10.0 ** rng.uniform(-4.0, -3.0))
        ra = float(10.0 ** rng.uniform(5.0, 6.0))
        dt = max([d for d in (1e-5, 2e-5, 5e-5, 1e-4) if d <= ek / 10.0] or [1e-5])
        out.append(RunSpec(run_id=i, l_max=l_max, n_r=n_r, ek=ek, ra=ra, dt=dt,
                           n_steps=n_steps, seed=1000 + i, arrival=t, precision=precision,
                           radial_scheme=radial_scheme))
    return out


def _grid_sizes(l_max, minc=1):
    """n_theta, n_phi and lm_max of the reference's grid derivation (params.py:57-76)."""
    n = 2 * ((30 * l_max) // 20)
    best, dmin = n, 1 << 30
    for i in range(0, 16):
        for j in range(0, 10):
            for k in range(0, 8):
                v = 2 ** i * 3 ** j * 5 ** k
                if 0 <= v - n < dmin:
                    dmin, best = v - n, v
    lm_max = sum(l_max - m + 1 for m in range(0, l_max + 1, minc))
    return best // 2, best // minc, lm_max


def footprint_estimate(spec):
    """Upper estimate of a run's device memory (bytes): 42 (lm_max, n_r) complex
    arrays (fields, time arrays, nonlinear outputs), the stage workspace
    (Fourier rows of 24 fields in FP64 and the split operand images), the
    solve operators (at most 8 (l_max + 1) n_r^2 doubles: the coupled (w, p)
    operators of the Chebyshev form are 2 n_r square) and the transform tables."""
    n_theta, n_phi, lm = _grid_sizes(spec.l_max)
    n_m = spec.l_max + 1
    arrays = 42 * lm * spec.n_r * 16
    fourier = 24 * spec.n_r * n_theta * n_m * 16
    images = (2 * 1.13e9 * (lm * spec.n_r) / (33024 * 97)) if spec.precision == "split" else 0
    ops = 8 * (spec.l_max + 1) * spec.n_r * (spec.n_r + 1) * 8
    tables = 8 * lm * (n_theta // 2) * 8
    return int(1.25 * (arrays + fourier + images + ops + tables)) + (64 << 20)


class GraphRunner:
    """One admitted run: a BoussinesqStep on its own stream, stepped by a CUDA
    graph captured after the first (eager) step.  cache: the server's shared
    read-only resources (transform plans, radial and solve operators per shape)."""

    def __init__(self, spec, device, use_graph=True, cache=None):
        from .step import BoussinesqStep

        self.spec = spec
        self.device = device
        self.stream = torch.cuda.Stream(device)
        self.inflight = []
        self.latencies_ms = []
        self.launched = 0
        self.graph = None
        with torch.cuda.stream(self.stream):
            self.st = BoussinesqStep(spec.l_max, spec.n_r, ek=spec.ek, ra=spec.ra, pr=spec.pr,
                                     prmag=spec.prmag, dt=spec.dt, precision=spec.precision,
                                     device=device, cache=cache,
                                     radial_scheme=spec.radial_scheme)
            self.st.init_random(seed=spec.seed, amp=spec.amp)
            self._launch(eager=True)
            if use_graph and spec.n_steps > 1:
                self.graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(self.graph, stream=self.stream):
                    self.st.step()

    def _launch(self, eager=False):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(self.stream):
            e0.record()
            if self.graph is not None and not eager:
                self.graph.replay()
            else:
                self.st.step()
            e1.record()
            if self.graph is not None and not eager:
                # a replay bypasses the plan's per-call watch: read the stage's
                # device status word after it, on the run's stream
                self.st.plan._watch(self.st.work, "nl_bouss (graph replay)", fused=True)
        self.inflight.append((e0, e1))
        self.launched += 1

    def launch(self):
        self._launch()

    def pending(self):
        return len(self.inflight)

    def poll(self):
        self.st.plan.poll_status()
        while self.inflight and self.inflight[0][1].query():
            e0, e1 = self.inflight.pop(0)
            self.latencies_ms.append(e0.elapsed_time(e1))

    def done(self):
        return self.launched >= self.spec.n_steps and not self.inflight

    def finish(self, keep_state=False):
        from .state import state_dict

        self.stream.synchronize()
        self.st.plan.poll_status(block=True)
        res = RunResult(self.spec, energies=self.st.energies(),
                        latencies_ms=list(self.latencies_ms))
        if keep_state:
            res.state = state_dict(self.st, step=self.spec.n_steps,
                                   sim_time=self.spec.n_steps * self.spec.dt)
        self.graph = None
        self.st = None
        return res


class EnsembleServer:
    """Continuous-batching loop over a run stream.

    budget_bytes: device memory the admitted runs may hold together (footprint
    estimates); max_active: slots; depth: steps each run keeps queued on its
    stream (graph replays are cheap to queue, and a deep queue keeps the GPU
    busy while the host builds the next admitted run)."""

    def __init__(self, device=None, budget_bytes=None, max_active=16, depth=64, use_graph=True,
                 runner=GraphRunner, footprint=footprint_estimate):
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget_bytes = int(0.8 * free)
        self.budget = int(budget_bytes)
        self.max_active, self.depth, self.use_graph = max_active, depth, use_graph
        self.runner, self.footprint = runner, footprint
        self.log = []  # (time s, event, run_id)
        # plans, radial operators and solve operators shared by runs of one shape
        # (the solve operators depend on the grid, dt, Pr and Pm only)
        self.cache = {}

    def serve(self, specs, keep_state=False, clock=time.perf_counter, sleep=time.sleep):
        pending = sorted(specs, key=lambda s: (s.arrival, s.run_id))
        for s in pending:
            if self.footprint(s) > self.budget:
                raise ValueError(f"run {s.run_id} needs {self.footprint(s)} bytes, budget "
                                 f"{self.budget}")
        active, results, used = [], [], 0
        t0 = clock()
        while pending or active:
            now = clock() - t0
            while (pending and pending[0].arrival <= now and len(active) < self.max_active
                   and used + self.footprint(pending[0]) <= self.budget):
                spec = pending.pop(0)
                used += self.footprint(spec)
                r = self.runner(spec, self.device, self.use_graph, self.cache)
                r.admitted_s = clock() - t0
                active.append(r)
                self.log.append((r.admitted_s, "admit", spec.run_id))
            busy = False
            for r in active:
                while r.launched < r.spec.n_steps and r.pending() < self.depth:
                    r.launch()
                    busy = True
            for r in list(active):
                r.poll()
                if r.done():
                    res = r.finish(keep_state)
                    res.admitted_s, res.finished_s = r.admitted_s, clock() - t0
                    results.append(res)
                    self.log.append((res.finished_s, "finish", r.spec.run_id))
                    active.remove(r)
                    used -= self.footprint(r.spec)
                    busy = True
            if not busy:
                if not active and pending:
                    sleep(max(0.0, min(0.01, pending[0].arrival - (clock() - t0))))
                else:
                    sleep(5e-5)
        self.wall_s = clock() - t0
        return sorted(results, key=lambda r: r.spec.run_id)


def latency_report(results, wall_s):
    """p50 / p99 per-step device latency (ms) over all steps of all runs, and the
    aggregate steps/s over the serving wall time."""
    lat = np.concatenate([np.asarray(r.latencies_ms, dtype=np.float64) for r in results]) \
        if results else np.zeros(0)
    steps = sum(r.spec.n_steps for r in results)
    return {"runs": len(results), "steps": steps,
            "p50_ms": float(np.percentile(lat, 50)) if lat.size else math.nan,
            "p99_ms": float(np.percentile(lat, 99)) if lat.size else math.nan,
            "steps_per_s": steps / wall_s if wall_s > 0 else math.nan, "wall_s": wall_s}


# ----------------------------------------------------------------------------
# Cross-run batching: one fused nonlinear stage for all runs of a resolution.


class _Member:
    def __init__(self, spec, st):
        self.spec, self.st = spec, st
        self.launched, self.latencies_ms = 0, []
        self.admitted_s = 0.0


def group_key(spec):
    """Runs that can share one stage launch: same horizontal grid (l_max),
    precision and magnetic Prandtl number (the stage's Courant factor depends on
    it); Ekman numbers may differ (the Lorentz factor is passed per level)."""
    return (spec.l_max, spec.precision, float(spec.prmag))


class GroupRunner:
    """The admitted runs of one group_key, stepped together.  A group step is:
    one mt_copy_levels launch gathering every member's eleven stage inputs into
    batch arrays whose radial levels are the members' levels side by side; one
    fused nonlinear stage over all of them (per-level Lorentz factor, profiles
    concatenated); one mt_copy_levels launch scattering the bulk levels of the
    eight outputs back into each member's nl_out; then each member's explicit
    terms and implicit solves.  Every kernel of the stage works per level (and
    the digit-split scales per row), so a run's result does not depend on the
    other members.  The group step is captured as one CUDA graph, captured again
    (after one eager step) whenever the membership changes; membership changes
    only when no group step is in flight."""

    def __init__(self, key, device, cache, use_graph=True, depth=8):
        self.key, self.device, self.cache = key, torch.device(device), cache
        self.use_graph, self.depth = use_graph, depth
        self.members, self.waiting = [], []
        self.inflight = []          # (e0, e1, members of that step)
        self.stream = torch.cuda.Stream(self.device)
        self.graph = None
        self.dirty = True
        self.launches = 0           # group steps launched
        self.kernels_per_step = 0   # library kernels per group step (gather, stage, scatter, per run)
        self.kernel_launches = 0    # library kernels over all group steps

    # membership ------------------------------------------------------------
    def add(self, spec, admitted_s=0.0):
        self.waiting.append((spec, admitted_s))

    def drained(self):
        return not self.inflight

    def active(self):
        return bool(self.members or self.waiting)

    def _join(self):
        from .step import BoussinesqStep

        with torch.cuda.stream(self.stream):
            for spec, t in self.waiting:
                st = BoussinesqStep(spec.l_max, spec.n_r, ek=spec.ek, ra=spec.ra, pr=spec.pr,
                                    prmag=spec.prmag, dt=spec.dt, precision=spec.precision,
                                    device=self.device, cache=self.cache,
                                    radial_scheme=spec.radial_scheme)
                st.init_random(seed=spec.seed, amp=spec.amp)
                m = _Member(spec, st)
                m.admitted_s = t
                self.members.append(m)
        self.waiting = []
        self.dirty = True

    def _build(self):
        """Batch arrays, level-copy descriptors and (after one eager step) the
        graph of the current membership."""
        from . import _lib
        from .step import BoussinesqStep

        ms = self.members
        dev = self.device
        plan = ms[0].st.plan
        lm = plan.lm_max
        n_tot = sum(m.st.n_r for m in ms)
        cd = torch.complex128
        self.b_in = {k: torch.zeros(lm, n_tot, dtype=cd, device=dev)
                     for k in BoussinesqStep.STAGE_INPUTS}
        self.b_out = {k: torch.zeros(lm, n_tot, dtype=cd, device=dev)
                      for k in BoussinesqStep.STAGE_OUTPUTS}
        self.b_prof = {k: torch.cat([m.st.prof[k] for m in ms]).contiguous()
                       for k in ("or2", "or4", "orho1", "orho2", "delxr2", "delxh2")}
        self.b_lf = torch.cat([torch.full((m.st.n_r,), m.st.LFfac, dtype=torch.float64,
                                          device=dev) for m in ms])
        self.b_work = torch.empty(plan.nl_bouss_workspace(n_tot, True, False), dtype=torch.uint8,
                                  device=dev)
        gather, scatter = [], []
        off = 0
        for m in ms:
            n = m.st.n_r
            for k in BoussinesqStep.STAGE_INPUTS:
                gather.append(_lib.LevelCopy(m.st.f[k].data_ptr(), self.b_in[k].data_ptr(), n,
                                             n_tot, 0, off, n, 0))
            for k in BoussinesqStep.STAGE_OUTPUTS:
                scatter.append(_lib.LevelCopy(self.b_out[k].data_ptr(), m.st.nl_out[k].data_ptr(),
                                              n_tot, n, off + 1, 1, n - 2, 0))
            off += n
        def to_dev(cps):
            arr = (_lib.LevelCopy * len(cps))(*cps)
            raw = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8)
            return raw.to(dev), len(cps)
        self.d_gather, self.n_gather = to_dev(gather)
        self.d_scatter, self.n_scatter = to_dev(scatter)
        self.plan, self.lm = plan, lm
        self.kernels_per_step = 2 + 6 + 6 * len(ms)
        self.graph = None
        self.dirty = False

    def _group_step(self):
        from . import _lib

        L = _lib.lib()
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(L.mt_copy_levels(self.lm, self.d_gather.data_ptr(), self.n_gather, s))
        ms = self.members
        opm = ms[0].st.opm
        self.plan.nl_bouss(self.b_in, self.b_prof, 0.0, 2.5, 1.0, opm, l_mag=True,
                           out=self.b_out, work=self.b_work, LFfac_r=self.b_lf)
        _lib.check(L.mt_copy_levels(self.lm, self.d_scatter.data_ptr(), self.n_scatter, s))
        for m in ms:
            m.st.explicit_terms()
            m.st.lm_loop()

    # stepping ---------------------------------------------------------------
    def can_launch(self):
        if not self.members or self.waiting or len(self.inflight) >= self.depth:
            return False
        return all(m.launched < m.spec.n_steps for m in self.members)

    def launch(self):
        eager = False
        if self.dirty:
            self._build()
            eager = True
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(self.stream):
            e0.record()
            if self.graph is not None and not eager:
                self.graph.replay()
            else:
                self._group_step()
            e1.record()
            if self.graph is not None and not eager:
                self.plan._watch(self.b_work, "nl_bouss (group graph replay)", fused=True)
        self.inflight.append((e0, e1, list(self.members)))
        for m in self.members:
            m.launched += 1
        self.launches += 1
        self.kernel_launches += self.kernels_per_step
        if eager and self.use_graph:
            with torch.cuda.stream(self.stream):
                self.stream.synchronize()
                self.graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(self.graph, stream=self.stream):
                    self._group_step()

    def poll(self):
        if self.members:
            self.members[0].st.plan.poll_status()
        while self.inflight and self.inflight[0][1].query():
            e0, e1, ms = self.inflight.pop(0)
            dt = e0.elapsed_time(e1)
            for m in ms:
                m.latencies_ms.append(dt)

    def retire(self, keep_state=False):
        """Finish the members that have done their steps (only when drained);
        admit the waiting runs.  Returns the finished RunResults."""
        from .state import state_dict

        if not self.drained():
            return []
        out = []
        done = [m for m in self.members if m.launched >= m.spec.n_steps]
        if done:
            self.stream.synchronize()
            done[0].st.plan.poll_status(block=True)
            for m in done:
                res = RunResult(m.spec, energies=m.st.energies(), latencies_ms=list(m.latencies_ms))
                if keep_state:
                    res.state = state_dict(m.st, step=m.spec.n_steps,
                                           sim_time=m.spec.n_steps * m.spec.dt)
                res.admitted_s = m.admitted_s
                out.append(res)
                self.members.remove(m)
            self.dirty = True
        if self.waiting:
            self._join()
        return out


class BatchedEnsembleServer:
    """Continuous batching with one fused stage per resolution group per step
    (GroupRunner): same admission rules as EnsembleServer (arrival, slots,
    memory budget); an admitted run joins its group at the group's next
    membership change (when no group step is in flight), and a finished run
    leaves it the same way."""

    def __init__(self, device=None, budget_bytes=None, max_active=16, depth=8, use_graph=True,
                 group_runner=GroupRunner, footprint=footprint_estimate):
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget_bytes = int(0.8 * free)
        self.budget = int(budget_bytes)
        self.max_active, self.depth, self.use_graph = max_active, depth, use_graph
        self.group_runner, self.footprint = group_runner, footprint
        self.log = []
        self.cache = {}
        self.groups = {}

    def serve(self, specs, keep_state=False, clock=time.perf_counter, sleep=time.sleep):
        pending = sorted(specs, key=lambda s: (s.arrival, s.run_id))
        for s in pending:
            if self.footprint(s) > self.budget:
                raise ValueError(f"run {s.run_id} needs {self.footprint(s)} bytes, budget "
                                 f"{self.budget}")
        results, used, n_active = [], 0, 0
        t0 = clock()
        while pending or any(g.active() for g in self.groups.values()):
            now = clock() - t0
            while (pending and pending[0].arrival <= now and n_active < self.max_active
                   and used + self.footprint(pending[0]) <= self.budget):
                spec = pending.pop(0)
                used += self.footprint(spec)
                n_active += 1
                key = group_key(spec)
                if key not in self.groups:
                    self.groups[key] = self.group_runner(key, self.device, self.cache,
                                                         self.use_graph, self.depth)
                self.groups[key].add(spec, now)
                self.log.append((now, "admit", spec.run_id))
            busy = False
            for g in self.groups.values():
                g.poll()
                for res in g.retire(keep_state):
                    res.finished_s = clock() - t0
                    results.append(res)
                    self.log.append((res.finished_s, "finish", res.spec.run_id))
                    used -= self.footprint(res.spec)
                    n_active -= 1
                    busy = True
                while g.can_launch():
                    g.launch()
                    busy = True
            if not busy:
                if not any(g.active() for g in self.groups.values()) and pending:
                    sleep(max(0.0, min(0.01, pending[0].arrival - (clock() - t0))))
                else:
                    sleep(5e-5)
        self.wall_s = clock() - t0
        return sorted(results, key=lambda r: r.spec.run_id)
