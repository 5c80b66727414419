"""Host logic of the ensemble serving loop (magic_b200.serve), on the CPU with
a stand-in runner and a virtual clock: admission only after arrival, within
the slot count and the memory budget; continuous batching (a run admitted
while others are still stepping); every run completes; the seeded run stream
follows the ensemble configuration's distributions."""

import numpy as np
import pytest

from magic_b200.serve import (EnsembleServer, RunResult, RunSpec, footprint_estimate,
                              latency_report, poisson_stream)


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-4)


class FakeRunner:
    """Each step takes `step_s` of virtual time after its launch; steps of one
    run are serial (stream order)."""
    clock = None
    step_s = 1e-3

    def __init__(self, spec, device, use_graph=True, cache=None):
        self.spec, self.launched, self.finish_times, self.latencies_ms = spec, 0, [], []
        self.launch()  # the eager first step, as GraphRunner does

    def launch(self):
        start = max([self.clock()] + self.finish_times[-1:])
        self.finish_times.append(start + self.step_s)
        self.launched += 1

    def pending(self):
        return sum(1 for t in self.finish_times if t > self.clock())

    def poll(self):
        pass

    def done(self):
        return self.launched >= self.spec.n_steps and self.pending() == 0

    def finish(self, keep_state=False):
        return RunResult(self.spec, latencies_ms=[self.step_s * 1e3] * self.spec.n_steps)


def _serve(specs, budget, max_active, fp):
    clock = Clock()
    FakeRunner.clock = clock
    srv = EnsembleServer(device="cpu", budget_bytes=budget, max_active=max_active,
                         runner=FakeRunner, footprint=fp)
    res = srv.serve(specs, clock=clock, sleep=clock.sleep)
    return srv, res


def _concurrency(log):
    cur, peak = 0, 0
    for _, ev, _ in sorted(log, key=lambda x: (x[0], x[1] == "admit")):
        cur += 1 if ev == "admit" else -1
        peak = max(peak, cur)
    return peak


def test_admission_respects_arrival_slots_and_budget():
    specs = [RunSpec(run_id=i, l_max=32, n_r=33, ek=1e-3, ra=1e5, n_steps=20, arrival=0.002 * i)
             for i in range(8)]
    fp = lambda s: 100
    srv, res = _serve(specs, budget=250, max_active=4, fp=fp)
    assert [r.spec.run_id for r in res] == list(range(8))
    admits = {rid: t for t, ev, rid in srv.log if ev == "admit"}
    for s in specs:
        assert admits[s.run_id] >= s.arrival
    assert _concurrency(srv.log) == 2            # budget 250 holds two runs of 100
    srv, _ = _serve(specs, budget=10 ** 9, max_active=3, fp=fp)
    assert _concurrency(srv.log) == 3            # now the slots limit


def test_continuous_batching_admits_while_others_run():
    specs = [RunSpec(run_id=0, l_max=32, n_r=33, ek=1e-3, ra=1e5, n_steps=200, arrival=0.0),
             RunSpec(run_id=1, l_max=32, n_r=33, ek=1e-3, ra=1e5, n_steps=10, arrival=0.05)]
    srv, res = _serve(specs, budget=10 ** 9, max_active=4, fp=lambda s: 1)
    t = {(ev, rid): tt for tt, ev, rid in srv.log}
    # run 1 arrives mid-way through run 0, is admitted at once and finishes first
    assert t[("admit", 1)] < t[("finish", 0)]
    assert t[("finish", 1)] < t[("finish", 0)]
    rep = latency_report(res, srv.wall_s)
    assert rep["steps"] == 210 and rep["p50_ms"] == pytest.approx(1.0)


def test_oversize_run_is_refused():
    specs = [RunSpec(run_id=0, l_max=32, n_r=33, ek=1e-3, ra=1e5)]
    with pytest.raises(ValueError):
        _serve(specs, budget=10, max_active=1, fp=lambda s: 100)


def test_poisson_stream_distributions():
    a = poisson_stream(64, rate=4.0, seed=3)
    b = poisson_stream(64, rate=4.0, seed=3)
    assert a == b
    arr = np.array([s.arrival for s in a])
    assert np.all(np.diff(arr) > 0) and 8.0 < arr[-1] < 32.0   # mean 16 s for 64 runs
    assert {s.l_max for s in a} <= {32, 64, 85, 127} and {s.n_r for s in a} <= {33, 49, 65}
    ek = np.array([s.ek for s in a])
    ra = np.array([s.ra for s in a])
    assert ek.min() >= 1e-4 and ek.max() <= 1e-3 and ra.min() >= 1e5 and ra.max() <= 1e6
    assert all(s.pr == 1.0 and s.prmag == 5.0 and s.amp == 1e-5 for s in a)


def test_footprint_grows_with_size():
    small = RunSpec(run_id=0, l_max=32, n_r=33, ek=1e-3, ra=1e5)
    big = RunSpec(run_id=1, l_max=127, n_r=65, ek=1e-3, ra=1e5)
    assert footprint_estimate(big) > 8 * footprint_estimate(small)


class FakeGroup:
    """Stand-in GroupRunner: a group step takes `step_s` of virtual time after
    the previous one; membership changes only when drained, as in GroupRunner."""
    clock = None
    step_s = 1e-3
    created = []

    def __init__(self, key, device, cache, use_graph=True, depth=8):
        self.key, self.depth = key, depth
        self.members, self.waiting, self.finish_times = [], [], []
        self.steps_with = []  # member run ids of every group step
        FakeGroup.created.append(self)

    def add(self, spec, admitted_s=0.0):
        self.waiting.append(spec)

    def _inflight(self):
        return sum(1 for t in self.finish_times if t > self.clock())

    def drained(self):
        return self._inflight() == 0

    def active(self):
        return bool(self.members or self.waiting)

    def can_launch(self):
        return (bool(self.members) and not self.waiting and self._inflight() < self.depth
                and all(m[1] < m[0].n_steps for m in self.members))

    def launch(self):
        start = max([self.clock()] + self.finish_times[-1:])
        self.finish_times.append(start + self.step_s)
        for m in self.members:
            m[1] += 1
        self.steps_with.append(tuple(m[0].run_id for m in self.members))

    def poll(self):
        pass

    def retire(self, keep_state=False):
        if not self.drained():
            return []
        done = [m for m in self.members if m[1] >= m[0].n_steps]
        for m in done:
            self.members.remove(m)
        out = [RunResult(m[0], latencies_ms=[self.step_s * 1e3] * m[0].n_steps) for m in done]
        self.members += [[s, 0] for s in self.waiting]
        self.waiting = []
        return out


def test_batched_server_groups_runs_and_admits_between_steps():
    from magic_b200.serve import BatchedEnsembleServer, group_key

    clock = Clock()
    FakeGroup.clock, FakeGroup.created = clock, []
    specs = [RunSpec(run_id=i, l_max=32 if i % 2 else 64, n_r=33, ek=1e-3 * (1 + i), ra=1e5,
                     n_steps=10 + i, arrival=0.003 * i) for i in range(8)]
    srv = BatchedEnsembleServer(device="cpu", budget_bytes=10 ** 9, max_active=8,
                                group_runner=FakeGroup, footprint=lambda s: 100)
    res = srv.serve(specs, clock=clock, sleep=clock.sleep)
    assert [r.spec.run_id for r in res] == list(range(8))
    # two resolution groups; every step of a group holds runs of that l_max only
    assert {g.key for g in FakeGroup.created} == {group_key(specs[0]), group_key(specs[1])}
    by_id = {s.run_id: s for s in specs}
    for g in FakeGroup.created:
        for ids in g.steps_with:
            assert {by_id[i].l_max for i in ids} == {g.key[0]}
    # every run took exactly its steps, and some group steps served several runs at once
    counts = {i: 0 for i in by_id}
    for g in FakeGroup.created:
        for ids in g.steps_with:
            for i in ids:
                counts[i] += 1
    assert counts == {i: by_id[i].n_steps for i in by_id}
    assert max(len(ids) for g in FakeGroup.created for ids in g.steps_with) >= 2
    admits = {rid: t for t, ev, rid in srv.log if ev == "admit"}
    for s in specs:
        assert admits[s.run_id] >= s.arrival


def test_group_key_separates_precision_and_pm():
    from magic_b200.serve import group_key

    a = RunSpec(run_id=0, l_max=32, n_r=33, ek=1e-3, ra=1e5)
    b = RunSpec(run_id=1, l_max=32, n_r=49, ek=5e-4, ra=3e5)
    c = RunSpec(run_id=2, l_max=32, n_r=33, ek=1e-3, ra=1e5, prmag=2.0)
    d = RunSpec(run_id=3, l_max=32, n_r=33, ek=1e-3, ra=1e5, precision="fp64")
    assert group_key(a) == group_key(b)
    assert len({group_key(x) for x in (a, c, d)}) == 3
