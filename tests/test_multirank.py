"""The N > 1 bench path on CPU ranks (gloo, world size 2): replicas integrate independent sweeps, the whole-job time
is the slowest rank's and the units add up."""
from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    t, n = bench.reduce_over_ranks(1.0 + rank, 100 * (rank + 1), dist, device="cpu")
    out[rank] = (t, n, bench.replica_seed("config2-block", rank))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_reduce_over_two_gloo_ranks():
    port = _free_port()
    manager = mp.get_context("spawn").Manager()     # no fork of a process that runs threads
    out = manager.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn")
    assert out[0][:2] == (2.0, 300) and out[1][:2] == (2.0, 300)
    assert out[0][2] != out[1][2]


def _replica_worker(rank, world, port, out):
    """One replica rank: plans its own sweep (the replica seed's crystal orientation and noise) with the CPU planner,
    integrates a few of its reflections with the CPU restatement, and reduces time and reflection count over ranks."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import time

    import numpy as np
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    import bench
    from oracle import kernels as OK
    from oracle import pipeline as OP
    from oracle.plan import plan_integration
    from xpg_b200 import synth
    from xpg_b200.plan import IntegrationModel
    t0 = time.perf_counter()
    spec = synth.config1(seed=bench.replica_seed("config1", rank), nframes=30)
    exp = spec.experiment()
    p = plan_integration([exp], np.array([0.0, 30.0]), IntegrationModel(spec.sigma_d, spec.sigma_m),
                         spec.resolution_limit(), 1e9, (1, 30), 0.05, spec.n_regions_xy, True, True)
    rows = np.flatnonzero((p.iz0 >= 0) & (p.iz0 + p.Dz * p.fb <= 30) & (p.pxs == 1))[:3]
    raw = synth.render_frames(spec, range(1, 31))
    prep = OP.prepared_frames(raw, 0, spec.overload, [1])
    g = exp.geom
    prof = np.repeat(OK.gaussian_profile()[None], p.nreg, 0)
    res = OP.integrate_rows(prep, list(range(30)), OP.row_payload(p, rows), OK.detector_consts(g, None),
                            g.s0.astype(np.float32), g.axis.astype(np.float32),
                            np.float32(np.radians(g.z_to_phi(0.0))), np.float32(np.radians(g.osc)),
                            np.radians(spec.sigma_d), np.radians(spec.sigma_m), 1.0, OK.rc_default_weights(), prof)
    t, n = bench.reduce_over_ranks(time.perf_counter() - t0, p.n, dist, device="cpu")
    out[rank] = (t, n, p.n, [float(o1["isum"]) for o1, _ in res], p.refl["hkl"][:5].tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_replica_ranks_plan_and_integrate_their_own_sweeps():
    """Two gloo ranks each plan and integrate (CPU restatement) their own replica sweep: the sweeps differ, the
    whole-job count is the sum of the ranks' reflections and the time the slowest rank's."""
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_replica_worker, args=(2, port, out), nprocs=2, start_method="spawn")
    t0, n0, own0, isum0, hkl0 = out[0]
    t1, n1, own1, isum1, hkl1 = out[1]
    assert n0 == n1 == own0 + own1 and t0 == t1
    assert hkl0 != hkl1 and len(isum0) == 3 and len(isum1) == 3
