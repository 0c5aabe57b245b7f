"""Batched and served integration (xpg_b200.batch): several sweeps in one scheduler, their completed blocks through
shared persistent pass-1 / pass-2 launches, each result the same bits as the sweep integrated alone."""
from __future__ import annotations

import numpy as np
import pytest

import golden_io as G

pytestmark = pytest.mark.gpu

KEYS = ("bg", "isum", "vsum", "vsum0", "iprf", "vprf", "vprf0", "corr", "xo", "yo", "zo", "p_valid", "p_total",
        "rho", "p_fg", "frac_rec", "m_d", "m_m", "n_over", "n_fg_masked", "isum_raw")
CASES = ("adaptive", "binned", "crowded", "superpix")


def _job(case):
    from xpg_b200 import frames as FR
    from xpg_b200.batch import Job
    from xpg_b200.plan import IntegrationModel
    z = G.load(case)
    spec, tmpl, mask, excl = G.case_inputs(case)
    edges = z["edges"]
    model = IntegrationModel(sigma_d=spec.sigma_d, sigma_m=spec.sigma_m, gain=1.0)
    kw = dict(frames=(1, spec.nframes), mask=mask, minimum_zeta=0.05, n_regions_xy=spec.n_regions_xy,
              exclude_frames=excl, bkg_template=tmpl, foreign_spots=G.foreign_of(case), wedge_frames=8)
    return Job(FR.U32Frames(G.frames_of(case), first=1, overload=spec.overload), [spec.experiment()] * (len(edges) - 1),
               edges, model, float(z["dmin"]), kw, label=case)


def _alone(job):
    from xpg_b200.integrate import integrate
    return integrate(job.images, job.exp_blocks, job.block_edges, job.model, job.dmin, verbose=False, **job.kwargs)


def _same(a, b, what):
    for k in KEYS:
        assert np.array_equal(np.asarray(a.refl[k]), np.asarray(b.refl[k]), equal_nan=True), (what, k)
    for blk in a.profiles:
        assert np.array_equal(a.profiles[blk], b.profiles[blk]), (what, blk)


def test_batched_results_equal_alone():
    from xpg_b200.batch import run_jobs
    jobs = [_job(c) for c in CASES]
    alone = [_alone(j) for j in jobs]
    res, stats = run_jobs(jobs)
    assert stats["rounds"] < stats["blocks"]              # blocks of several sweeps shared rounds
    for c, a, b in zip(CASES, alone, res):
        _same(a, b, c)


def test_admission_by_memory_keeps_results():
    """A budget that holds one sweep at a time: sweeps wait and are admitted as memory frees up, same results."""
    from xpg_b200.batch import job_footprint, run_jobs
    jobs = [_job(c) for c in ("adaptive", "binned")]
    alone = [_alone(j) for j in jobs]
    need = [job_footprint(j) for j in jobs]
    res, stats = run_jobs(jobs, budget_bytes=max(need) + min(need) // 2)     # one at a time, none split
    assert all(r.memory["parts"] == 1 for r in res)
    assert stats["admitted_at"][1] >= stats["admitted_at"][0]
    for c, a, b in zip(("adaptive", "binned"), alone, res):
        _same(a, b, c)


def test_served_results_equal_alone_and_latency_recorded():
    """Requests whose wedges arrive over time (interleaved sweeps, jittered arrivals): every wedge's latency is
    recorded and each sweep's results are the same alone and in the mix."""
    from xpg_b200.batch import serve
    rng = np.random.default_rng(3)
    jobs = [_job(c) for c in CASES]
    alone = [_alone(j) for j in jobs]
    for k, j in enumerate(jobs):
        nw = len(range(1, j.kwargs["frames"][1] + 1, j.kwargs["wedge_frames"]))
        j.arrivals = 0.01 * k + np.cumsum(rng.exponential(0.004, nw))
    res, stats = serve(jobs)
    n_wedges = sum(len(j.arrivals) for j in jobs)
    assert len(stats["latency"]) == n_wedges
    assert all(lat >= 0 for _, _, lat in stats["latency"])
    for c, a, b in zip(CASES, alone, res):
        _same(a, b, c)


def test_served_slots_plan_each_sweep_in_its_share():
    """slots: every sweep is planned for budget / slots (its blocks in parts when its open blocks exceed that share;
    live frames take no second pass), so that the sweeps run together; each result is the same as the sweep
    integrated alone under that share."""
    from xpg_b200.batch import job_footprint, serve
    from xpg_b200.integrate import integrate
    cases = ("adaptive", "crowded")
    jobs = [_job(c) for c in cases]
    need = [job_footprint(j) for j in jobs]
    share = 0.7 * min(need)
    for j in jobs:
        j.images.rereadable = False
    alone = [integrate(j.images, j.exp_blocks, j.block_edges, j.model, j.dmin, verbose=False, mem_budget=share,
                       **j.kwargs) for j in jobs]
    assert any(a.memory["parts"] > 1 for a in alone)
    rng = np.random.default_rng(5)
    for k, j in enumerate(jobs):
        nw = len(range(1, j.kwargs["frames"][1] + 1, j.kwargs["wedge_frames"]))
        j.arrivals = 0.005 * k + np.cumsum(rng.exponential(0.004, nw))
    res, stats = serve(jobs, budget_bytes=2 * share, slots=2)
    assert stats["admitted_at"][1] <= j.arrivals[0] + 0.5            # both sweeps ran at once
    for c, a, b in zip(cases, alone, res):
        assert b.memory["parts"] == a.memory["parts"] and "passes" not in b.memory
        _same(a, b, c)


def test_concurrent_results_equal_alone():
    """Sweeps integrated on three host threads at once (each the plain path on streams of its own, sharing the
    device and the buffer pool): the same bits as each sweep integrated alone."""
    from xpg_b200.batch import integrate_concurrent
    jobs = [_job(c) for c in CASES]
    alone = [_alone(j) for j in jobs]
    res, stats = integrate_concurrent(jobs, workers=3)
    assert len(stats["admitted_at"]) == len(jobs)
    for c, a, b in zip(CASES, alone, res):
        _same(a, b, c)
