"""Host logic of the plan's device-status watch: which calls record their
workspace's status word (the first int, written by a bounded tensor-pipe wait
that ran out).  Split plans record every call; digit-split (ozaki) plans only
the fused stages (nl_bouss, nl_anel), whose digit-plane GEMMs carry the bounded
waits; FP64 plans only the fused stages too (their kernels leave the word
alone, so it reads 0)."""

import inspect

from magic_b200.plan import Plan


class _Rec:
    def __init__(self):
        self.seen = []

    def record(self, work, what):
        self.seen.append(what)


def _plan(precision):
    p = object.__new__(Plan)  # no device plan: only the watch's decision
    p._h = None
    p._status = _Rec()
    p.precision = precision
    return p


def test_split_plans_watch_every_call():
    p = _plan("split")
    p._watch(None, "scal_to_spat")
    p._watch(None, "nl_anel", fused=True)
    assert p._status.seen == ["scal_to_spat", "nl_anel"]


def test_digit_split_plans_watch_the_fused_stages():
    p = _plan("ozaki")
    p._watch(None, "scal_to_spat")
    p._watch(None, "nl_bouss", fused=True)
    p._watch(None, "nl_anel", fused=True)
    assert p._status.seen == ["nl_bouss", "nl_anel"]


def test_fused_stage_calls_mark_themselves_fused():
    for name in ("nl_bouss", "nl_anel"):
        src = inspect.getsource(getattr(Plan, name))
        assert f'self._watch(work, "{name}", fused=True)' in src, name
