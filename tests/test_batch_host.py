"""Host logic of the concurrent many-sweep form (xpg_b200.batch.integrate_concurrent) without a GPU: planned runs and
the frame loop replaced by fakes that record when they run. Sweeps start only while their planned peaks fit the
budget together (a sweep larger than the budget runs alone), every sweep runs once and is closed, results come back
in job order, and a failing sweep's error reaches the caller."""
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
