"""Host logic of the many-sweep schedulers (xpg_b200.batch) without a GPU, the planned runs replaced by fakes that
record their stages.

integrate_concurrent: sweeps start only while their planned peaks fit the budget together (a sweep larger than the
budget runs alone), every sweep runs once and is closed, results come back in job order, and a failing sweep's error
reaches the caller. run_jobs (batched and served): every block of every sweep goes through pass 1, learning and
pass 2 in its sweep's order, blocks of several sweeps share rounds, a sweep planned in two passes over the frames
is fed twice, and served wedges are fed no earlier than their arrival, each with a latency."""
from __future__ import annotations

import contextlib
import importlib
import threading
import time

import pytest

from xpg_b200 import batch as B

I = importlib.import_module("xpg_b200.integrate")         # the module (the package exports the function by this name)


class _Job:
    def __init__(self, label, need, seconds, fail=False):
        self.label, self.need, self.seconds, self.fail = label, need, seconds, fail
        self.images = self                     # the fake run finds its job through the frames argument
        self.exp_blocks = self.block_edges = self.model = self.dmin = None
        self.kwargs = {}


@pytest.fixture
def log(monkeypatch):
    rec = dict(live=0, used=0, max_used=0, max_live=0, runs=[], closed=0)
    lock = threading.Lock()

    class FakeRun:
        def __init__(self, images, *a, **kw):
            self.job = images
            self.mem = {"peak": images.need}

        def close(self):
            with lock:
                rec["closed"] += 1

    def fake_drive(run):
        with lock:
            rec["live"] += 1
            rec["used"] += run.job.need
            rec["max_live"] = max(rec["max_live"], rec["live"])
            rec["max_used"] = max(rec["max_used"], rec["used"])
            rec["runs"].append(run.job.label)
        try:
            time.sleep(run.job.seconds)
            if run.job.fail:
                raise RuntimeError("sweep failed: " + run.job.label)
            return "result " + run.job.label
        finally:
            with lock:
                rec["live"] -= 1
                rec["used"] -= run.job.need

    @contextlib.contextmanager
    def no_stream(device):
        yield None

    monkeypatch.setattr(B, "SweepRun", FakeRun)
    monkeypatch.setattr(I, "drive", fake_drive)
    monkeypatch.setattr(B, "_own_stream", no_stream)
    return rec


def test_admission_keeps_planned_peaks_within_budget(log):
    jobs = [_Job(f"s{k}", need, 0.05) for k, need in enumerate((40, 30, 50, 20, 60, 10))]
    res, stats = B.integrate_concurrent(jobs, budget_bytes=100, workers=3, device="cpu")
    assert res == [f"result s{k}" for k in range(6)]
    assert sorted(log["runs"]) == sorted(j.label for j in jobs)
    assert log["max_used"] <= 100 and log["max_live"] >= 2          # sweeps overlapped, within the budget
    assert stats["peak_bytes"] <= 100 and len(stats["admitted_at"]) == 6
    assert log["closed"] == 6


def test_a_sweep_larger_than_the_budget_runs_alone(log):
    jobs = [_Job("big", 250, 0.05), _Job("a", 30, 0.05), _Job("b", 30, 0.05)]
    res, _ = B.integrate_concurrent(jobs, budget_bytes=100, workers=3, device="cpu")
    assert res == ["result big", "result a", "result b"]
    assert log["max_used"] <= 250 and log["closed"] == 3
    if log["max_used"] > 100:                                        # "big" ran, and ran alone
        assert log["max_live"] >= 1


def test_a_failing_sweep_raises(log):
    jobs = [_Job("ok", 10, 0.01), _Job("bad", 10, 0.01, fail=True)]
    with pytest.raises(RuntimeError, match="sweep failed: bad"):
        B.integrate_concurrent(jobs, budget_bytes=100, workers=2, device="cpu")
    assert log["closed"] == 2 and log["live"] == 0


# ---- the batched / served scheduler (run_jobs) with fake runs -----------------------------------------------------

class _Rows:
    def __init__(self, n):
        import numpy as np
        self.n = n
        self.bx = np.full(n, 17, np.int32)
        self.Dz = np.full(n, 9, np.int32)


class _Blk:
    def __init__(self, n):
        self.rowset = _Rows(n)


class FakeSweep:
    """A sweep of n_wedges wedges whose block k opens at wedge 2k and completes at wedge 2k + 1, in n_passes passes
    over the frames (block k in pass k % n_passes); records every stage call."""

    registry = []

    def __init__(self, images, *a, mem_budget=None, **kw):
        import numpy as np
        self.job = images
        self.spec = images.spec
        self.wedges = [(f, f) for f in range(self.spec["wedges"])]
        self.n_passes = self.spec.get("passes", 1)
        self.pass_index = 0
        self.mem = {"peak": self.spec["need"]}
        self.device = "cpu"
        self.last_gathered = None
        self.opened, self.live, self.reported = {}, {}, set()
        self.calls = []
        self.blocks = [k for k in range(self.spec["wedges"] // 2)]
        self.done = []
        self.closed = False
        FakeSweep.registry.append(self)
        self._np = np

    def _mine(self, b):
        return b % self.n_passes == self.pass_index

    def feed(self, w):
        self.calls.append(("feed", self.pass_index, w))
        if w % 2 == 0 and w // 2 in self.blocks and self._mine(w // 2):
            self.opened[w // 2] = _Blk(5)
        out = [b for b in list(self.opened) if 2 * b + 1 <= w and b not in self.reported]
        self.reported.update(out)
        return out

    def remaining(self):
        out = [b for b in self.opened if b not in self.reported]
        self.reported.update(out)
        return out

    def pass1_stage(self, b, batched=False):
        self.live[b] = self.opened.pop(b)
        self.calls.append(("pass1", b))
        return ("set", b), self._np.arange(self.live[b].rowset.n)

    def learn(self, b):
        self.calls.append(("learn", b))

    def pass2_stage(self, b, batched=False):
        self.calls.append(("pass2", b))
        return ("set2", b)

    def collect(self, b):
        self.live.pop(b)
        self.done.append((self.pass_index, b))

    def start_pass(self, k):
        self.pass_index = k
        self.reported = set()

    def result(self):
        return ("result", self.job.label, tuple(sorted(self.done)))

    def close(self):
        self.closed = True


class _Src:
    def __init__(self, label, **spec):
        self.label, self.spec = label, spec


def _jobs(specs, arrivals=None):
    out = []
    for k, (label, spec) in enumerate(specs):
        src = _Src(label, **spec)
        j = B.Job(src, [None], None, None, None, {}, label=label)
        if arrivals is not None:
            j.arrivals = arrivals[k]
        out.append(j)
    return out


@pytest.fixture
def fake_sched(monkeypatch):
    class FakeD:
        @staticmethod
        def RowSetTable(sets, dev):
            return list(sets)

        @staticmethod
        def batched_items(groups, bins, dev):
            return groups

        @staticmethod
        def pass1_batched(table, items):
            pass

        @staticmethod
        def pass2_batched(table, items):
            pass

    class FakeEvent:
        def record(self, stream=None):
            pass

        def query(self):
            return True

    FakeSweep.registry = []
    monkeypatch.setattr(B, "SweepRun", FakeSweep)
    monkeypatch.setattr(B, "D", FakeD)
    monkeypatch.setattr(B.torch.cuda, "Event", FakeEvent)
    return FakeSweep.registry


def test_run_jobs_processes_every_block_in_order_and_admits_by_budget(fake_sched):
    jobs = _jobs([("a", dict(wedges=8, need=60)), ("b", dict(wedges=6, need=50)), ("c", dict(wedges=4, need=30))])
    res, stats = B.run_jobs(jobs, budget_bytes=100, device="cpu")
    assert [r[1] for r in res] == ["a", "b", "c"]
    assert [r[2] for r in res] == [tuple((0, b) for b in range(n)) for n in (4, 3, 2)]
    assert stats["peak_bytes"] <= 100 + 60                   # a sweep is admitted alone even when it is large
    assert stats["admitted_at"][1] >= stats["admitted_at"][0]
    assert all(s.closed for s in fake_sched)
    for s in fake_sched:                                      # pass 1, learning and pass 2 in block order
        p1 = [c[1] for c in s.calls if c[0] == "pass1"]
        assert p1 == sorted(p1)
    assert stats["blocks"] == 9 and stats["rounds"] < stats["blocks"]   # blocks of several sweeps shared rounds


def test_run_jobs_restarts_the_frames_for_a_second_pass(fake_sched):
    jobs = _jobs([("a", dict(wedges=8, need=10, passes=2))])
    res, _ = B.run_jobs(jobs, budget_bytes=100, device="cpu")
    assert res[0][2] == ((0, 0), (0, 2), (1, 1), (1, 3))       # even blocks in pass 0, odd ones in pass 1
    feeds = [c for c in fake_sched[0].calls if c[0] == "feed"]
    assert [c[2] for c in feeds] == list(range(8)) * 2 and {c[1] for c in feeds} == {0, 1}


def test_served_wedges_wait_for_their_arrival_and_each_has_a_latency(fake_sched):
    import numpy as np
    arrivals = [np.array([0.0, 0.02, 0.04, 0.06]), np.array([0.01, 0.03, 0.05, 0.07])]
    jobs = _jobs([("a", dict(wedges=4, need=10)), ("b", dict(wedges=4, need=10))], arrivals)
    fed_at = []
    clock = time.perf_counter
    t0 = clock()
    orig_feed = FakeSweep.feed

    def timed_feed(self, w):
        fed_at.append((self.job.label, w, clock() - t0))
        return orig_feed(self, w)
    FakeSweep.feed = timed_feed
    try:
        res, stats = B.run_jobs(jobs, budget_bytes=100, device="cpu", served=True)
    finally:
        FakeSweep.feed = orig_feed
    arr = {("a", w): arrivals[0][w] for w in range(4)}
    arr.update({("b", w): arrivals[1][w] for w in range(4)})
    assert all(t >= arr[(lab, w)] - 0.005 for lab, w, t in fed_at)       # never fed before it arrived
    assert len(stats["latency"]) == 8 and all(lat >= 0 for _, _, lat in stats["latency"])
    assert [r[1] for r in res] == ["a", "b"]
