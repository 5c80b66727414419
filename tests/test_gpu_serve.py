"""The ensemble serving loop on the GPU: runs of different l_max, n_r, Ekman
and Rayleigh numbers served together (two of them sharing a plan and the solve
operators) give, bit for bit, the results they give alone; the CUDA-graph steps give the eager steps' results; the largest run of
the ensemble configuration (l_max = 127, 65 levels) is served in split
precision beside smaller ones."""

import pytest
import torch

pytestmark = pytest.mark.gpu


def _spec(i, l_max, n_r, arrival=0.0, steps=12):
    from magic_b200.serve import RunSpec

    return RunSpec(run_id=i, l_max=l_max, n_r=n_r, ek=10 ** (-3.0 - 0.3 * i),
                   ra=10 ** (5.0 + 0.4 * i), n_steps=steps, seed=10 + i, amp=1e-5,
                   arrival=arrival)


def _serve(specs, **kw):
    from magic_b200.serve import EnsembleServer

    srv = EnsembleServer(budget_bytes=40 << 30, **kw)
    return {r.spec.run_id: r for r in srv.serve(specs, keep_state=True)}, srv


def _same(a, b):
    for k, v in a.items():
        if torch.is_tensor(v):
            assert torch.equal(v, b[k]), k


def test_result_same_alone_and_in_the_mix():
    A = _spec(0, 32, 33)
    alone, _ = _serve([A])
    # run 3 has run 0's shape: the two share the plan and the solve operators
    mix, srv = _serve([A, _spec(1, 64, 49, arrival=0.0), _spec(2, 127, 65, arrival=0.001),
                       _spec(3, 32, 33, arrival=0.002)])
    admits = [rid for _, ev, rid in srv.log if ev == "admit"]
    finishes = [t for t, ev, _ in srv.log if ev == "finish"]
    assert len(admits) == 4 and max(t for t, ev, _ in srv.log if ev == "admit") < min(finishes)
    assert sum(1 for k in srv.cache if k[0] == "plan") == 3
    _same(alone[0].state, mix[0].state)
    for r in mix.values():
        ek, em = r.energies
        assert all(torch.isfinite(torch.tensor(list(ek) + list(em))))
        assert len(r.latencies_ms) == r.spec.n_steps


def test_graph_steps_equal_eager_steps():
    A = _spec(3, 64, 33, steps=8)
    g, _ = _serve([A], use_graph=True)
    e, _ = _serve([A], use_graph=False)
    _same(g[3].state, e[3].state)


@pytest.mark.parametrize("precision", ["split", "ozaki", "fp64"])
def test_batched_result_same_alone_and_in_the_mix(precision):
    """Cross-run batching: runs of one l_max share one fused stage per step (their
    levels side by side, per-level Lorentz factor), joining and leaving the group
    as they arrive and finish; each run's final state equals, bit for bit, its
    state when served alone (every stage kernel works per level and per row)."""
    import dataclasses

    from magic_b200.serve import BatchedEnsembleServer, EnsembleServer

    specs = [dataclasses.replace(s, precision=precision) for s in
             (_spec(0, 32, 33, steps=10), _spec(1, 32, 49, arrival=0.0, steps=14),
              _spec(2, 64, 33, arrival=0.0, steps=9), _spec(3, 32, 33, arrival=0.001, steps=7))]
    alone = {}
    for s in specs:
        srv = EnsembleServer(budget_bytes=40 << 30)
        alone[s.run_id] = srv.serve([s], keep_state=True)[0]
    bsrv = BatchedEnsembleServer(budget_bytes=40 << 30)
    mix = {r.spec.run_id: r for r in bsrv.serve(specs, keep_state=True)}
    assert sorted(mix) == [0, 1, 2, 3]
    g32 = bsrv.groups[(32, precision, 5.0)]
    assert g32.launches < sum(s.n_steps for s in specs if s.l_max == 32)  # steps were shared
    for i, r in mix.items():
        assert len(r.latencies_ms) == r.spec.n_steps
        _same(alone[i].state, r.state)
