"""The forward-model likelihood passes on the device (xpg_b200.forward: xi_fm_scatter / xi_fm_gather, the drop-in
for XPG's xpg/forward/kernels.py) against XPG's own passes on the same inputs (tests/golden/forward.npz) and the
oracle, through the C ABI. Float sums in another order: within 1e-5 of the value's scale (tests/test_forward.py)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import forward as OF
from test_forward import RTOL, cases

pytestmark = pytest.mark.gpu


class _Win:
    def __init__(self, w):
        self.f0, self.f1, self.y0, self.ny, self.x0, self.nx = (int(v) for v in w)


def _t(a, dt=None):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt).cuda()


@pytest.mark.parametrize("ns_dtype", [torch.int16, torch.int32, torch.float32])
def test_device_passes_match_xpg_and_oracle(ns_dtype):
    from xpg_b200 import forward as F
    for c in cases():
        win = _Win(c["win"])
        n = int(c["n"])
        beta = c["beta"] if c["beta"].size else None
        mu = _t(c["B"])
        M, A, NS = _t(c["M"]), _t(c["A"]), _t(c["NS"], ns_dtype)
        g0 = torch.zeros(n, dtype=torch.float32, device="cuda")
        g1 = torch.zeros_like(g0)
        fd = torch.zeros_like(g0)
        for grp in c["groups"]:
            R, P = _t(grp["R"]), _t(grp["P"])
            iz0, iy0, ix0 = _t(grp["iz0"]), _t(grp["iy0"]), _t(grp["ix0"])
            rows = _t(grp["rows"])
            F.scatter(mu, R, P, _t(c["I"][grp["rows"]]), _t(beta[grp["rows"]]) if beta is not None else None,
                      iz0, iy0, ix0, win)
            F.gather(g0, None, R, P, rows, iz0, iy0, ix0, win, A, M, NS, 0)
            F.gather(g1, fd, R, P, rows, iz0, iy0, ix0, win, None, M, NS, 1)
        torch.cuda.synchronize()
        got = dict(mu=mu.cpu().numpy(), gr=g0.cpu().numpy(), gn=g1.cpu().numpy(), fd=fd.cpu().numpy())
        ora_mu = OF.scatter(c["B"], c["groups"], c["I"], beta, c["win"])
        ora_gr, _ = OF.gather(c["groups"], c["win"], n, c["A"], c["M"], c["NS"], 0)
        ora_gn, ora_fd = OF.gather(c["groups"], c["win"], n, None, c["M"], c["NS"], 1)
        for key, ours, xpg, ora, floor in (("mu", got["mu"], c["xpg_mu"], ora_mu, 1.0),
                                           ("gr", got["gr"], c["xpg_grad_ratio"], ora_gr, 1e-3),
                                           ("gn", got["gn"], c["xpg_grad_newton"], ora_gn, 1e-3),
                                           ("fd", got["fd"], c["xpg_fisher_diag"], ora_fd, 1e-3)):
            scale = np.maximum(np.abs(ora), floor)
            assert (np.abs(ours - ora) <= RTOL * scale).all(), key
            assert (np.abs(ours - xpg) <= RTOL * scale).all(), key


def test_empty_chunk_and_argument_checks():
    from xpg_b200 import forward as F
    win = _Win([0, 4, 0, 8, 0, 8])
    mu = torch.zeros(4 * 64, dtype=torch.float32, device="cuda")
    R = torch.zeros((1, 0, 3), dtype=torch.float32, device="cuda")
    P = torch.zeros((1, 0, 5, 5), dtype=torch.float32, device="cuda")
    e = torch.zeros(0, dtype=torch.int64, device="cuda")
    assert F.scatter(mu, R, P, torch.zeros(0, device="cuda"), None, e, e, e, win) is mu
    R1 = torch.zeros((1, 1, 3), dtype=torch.float64, device="cuda")
    P1 = torch.zeros((1, 1, 5, 5), dtype=torch.float32, device="cuda")
    o = torch.zeros(1, dtype=torch.int64, device="cuda")
    with pytest.raises(TypeError):                     # float32 factors only
        F.scatter(mu, R1, P1, torch.zeros(1, device="cuda"), None, o, o, o, win)
    with pytest.raises(ValueError):                    # R and P disagree on the reflections
        F.scatter(mu, R1.float(), P1[:, :0].contiguous(), torch.zeros(1, device="cuda"), None, o, o, o, win)
