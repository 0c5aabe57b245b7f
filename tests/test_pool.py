"""The device buffer pool's reuse rule (xpg_b200.device.BufferPool), on host tensors: a request takes the smallest
kept buffer that holds it and is at most FIT times its size; a kept buffer much larger stays for a larger request."""
from __future__ import annotations

import torch

from xpg_b200.device import BufferPool


def test_pool_reuses_buffers_of_about_the_size_asked():
    pool = BufferPool()
    a = pool.take(100_000, torch.float32, "cpu")
    assert a.numel() == 100_000 and a._base.numel() == int(100_000 * pool.SLACK)
    base = a._base
    pool.give(a)
    b = pool.take(90_000, torch.float32, "cpu")            # within FIT: the kept buffer
    assert b._base is base and b.numel() == 90_000
    pool.give(b)
    c = pool.take(20_000, torch.float32, "cpu")            # far smaller: a new buffer, the large one stays kept
    assert c._base is not base
    assert any(t is base for t in pool.free[(None, torch.float32)])
    d = pool.take(100_000, torch.float32, "cpu")           # the large request takes it
    assert d._base is base
    pool.give(c)
    pool.give(d)
    e = pool.take(200_000, torch.float32, "cpu")           # larger than every kept one: those smaller are dropped
    assert e._base is not base and not pool.free[(None, torch.float32)]
    pool.clear()
    assert not pool.free


def test_pool_retains_only_buffers_a_run_can_take():
    pool = BufferPool()
    a = pool.take(100_000, torch.float32, "cpu")
    b = pool.take(10_000, torch.float32, "cpu")
    c = pool.take(5_000, torch.uint8, "cpu")
    pool.give(a)
    pool.give(b)
    pool.give(c)
    pool.retain({torch.float32: [95_000]})            # the next run's arenas: about a's size; no uint8 request
    kept = pool.free[(None, torch.float32)]
    assert len(kept) == 1 and kept[0] is a._base
    assert not pool.free[(None, torch.uint8)]
