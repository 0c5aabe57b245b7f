"""GPU parity of the pass-1 / accumulation / pass-2 kernels, called through the C ABI (libxpgi.so), on the shoebox
chunks stored in the golden fixtures: against the oracle (same arithmetic contract: integers and per-pixel terms
bit-exact, sums to float64-rounding) and against the reference's own outputs (tolerance.py)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import golden_io as G
import tolerance as T
from oracle import kernels as OK

pytestmark = pytest.mark.gpu

CASES = G.CASES


def _rows_from_chunk(d, rc, nb, device):
    from xpg_b200 import device as D
    m, Dz, Dy, Dx = d["sb"].shape
    pxs = rc["pxs"].astype(np.int32) if "pxs" in rc else np.ones(m, np.int32)
    return D.RowSet(S=rc["S"], phi=rc["phi"], ix0=rc["ix0"], iy0=rc["iy0"], iz0=rc["iz0"], fb=rc["fb"],
                    region=rc["region"], has_p=rc["has_p"], pS=rc["pS"], pphi=rc["pphi"], pxs=pxs,
                    Dz=np.full(m, Dz), bx=np.full(m, Dx), nb=nb, device=device, sb_bias=0.0)


def _block(d, prefix=""):
    from xpg_b200 import native as N
    b = N.XiBlock()
    b.frames_phi0 = float(d["frames_phi0"])
    b.osc = float(d["osc"])
    b.sd = float(d[prefix + "sd"])
    b.sm = float(d[prefix + "sm"])
    b.gain = float(d[prefix + "gain"])
    rcw = torch.as_tensor(np.asarray(d[prefix + "rcw"], np.float32)).cuda()
    b.rcw = N.ptr(rcw)
    for c in range(3):
        b.s0[c] = float(d["s0"][c])
        b.axis[c] = float(d["axis"][c])
    return b, rcw


def _run_case(case):
    from xpg_b200 import device as D
    spec, tmpl, mask, excl = G.case_inputs(case)
    g = spec.geometry()
    det = D.DeviceDetector(g, tmpl)
    odet = OK.detector_consts(g, tmpl)
    results = []
    for i in G.chunks(case):
        d, rc, nb, o1, o2 = G.chunk(case, i)
        rows = _rows_from_chunk(d, rc, nb, "cuda")
        arena = torch.as_tensor(d["sb"].reshape(-1)).cuda()
        blk, keep = _block(d)
        p1 = D.Pass1Buffers(rows)
        D.pass1(det, rows, blk, arena, p1)
        D.status()
        h1 = {k: v.cpu().numpy() for k, v in p1.t.items()}
        res = dict(chunk=i, d=d, rc=rc, nb=nb, o1=o1, o2=o2, rows=rows, h1=h1, odet=odet)
        if o2:
            prof = torch.as_tensor(d["prof"]).cuda()
            blk2, keep2 = _block(d, "p2_")
            p2 = D.Pass2Buffers(rows)
            D.pass2(det, rows, blk2, arena, prof, p1, p2)
            D.status()
            res["h2"] = {k: v.cpu().numpy() for k, v in p2.t.items()}
        results.append(res)
    return results


def _row_out(h1, rows, j):
    """Row j's pass-1 outputs in the oracle's shapes."""
    Dz, bx = int(rows.Dz[j]), int(rows.bx[j])
    po, fo = rows.pix_off[j], rows.frm_off[j]
    o = {k: h1[k][j] for k in h1 if h1[k].shape[0] == rows.n}
    for k in ("img2", "J", "u1", "u2", "all_valid2"):
        o[k] = h1[k][po:po + bx * bx].reshape(bx, bx)
    o["all_valid2"] = o["all_valid2"].astype(bool)
    o["fz"] = h1["fz"][fo:fo + Dz]
    return o


@pytest.fixture(scope="module", params=CASES)
def case_results(request):
    return request.param, _run_case(request.param)


EXACT = ("n_over", "n_fg_masked", "n_fg_nb", "nfg", "isum_raw", "bg", "nbg", "zeta", "seff", "all_valid2", "J", "u1",
         "u2")


def test_pass1_matches_oracle(case_results):
    """Integer counts, masks, the background and every per-pixel geometric term are bit-exact with the oracle; the
    accumulated sums (float32 within a pixel column, float64 across columns on the device; float64 throughout in
    the oracle) agree within 1e-5 of their scale."""
    case, results = case_results
    for r in results:
        d, rc, nb = r["d"], r["rc"], r["nb"]
        for j in range(r["rows"].n):
            mine = _row_out(r["h1"], r["rows"], j)
            ref = OK.pass1(d["sb"][j], G.row_dict(rc, j), G.nb_row(nb, j), r["odet"], d["s0"], d["axis"],
                           d["frames_phi0"], d["osc"], d["sd"], d["sm"], d["gain"], d["rcw"])
            for k in EXACT:
                a, b = np.asarray(mine[k]), np.asarray(ref[k])
                assert np.array_equal(a.astype(np.float64), b.astype(np.float64)), (case, r["chunk"], j, k)
            for k in ("isum", "vsum", "vsum0", "xo", "yo", "zo", "m_d", "m_m", "frac_rec", "img2", "fz"):
                ok, worst = T.within(k, mine[k], ref[k], ref, rel=1e-5)
                assert ok, (case, r["chunk"], j, k, worst)


def test_pass1_matches_reference(case_results):
    """Against XPG's own pass 1: integers exact, floats within tolerance.py."""
    case, results = case_results
    for r in results:
        o1 = r["o1"]
        for j in range(r["rows"].n):
            mine = _row_out(r["h1"], r["rows"], j)
            ctx = {k: o1[k][j] for k in o1}
            for k in ("n_over", "n_fg_masked", "n_fg_nb", "nfg"):
                assert int(mine[k]) == int(o1[k][j]), (case, r["chunk"], j, k)
            assert np.array_equal(mine["all_valid2"], o1["all_valid2"][j]), (case, r["chunk"], j)
            for k in ("bg", "nbg", "isum", "vsum", "vsum0", "xo", "yo", "zo", "m_d", "m_m", "frac_rec", "zeta",
                      "seff", "J", "u1", "u2", "img2", "fz"):
                ok, worst = T.within(k, mine[k], o1[k][j], ctx)
                assert ok, (case, r["chunk"], j, k, worst)


def test_pass2_matches_oracle_and_reference(case_results):
    case, results = case_results
    n = 0
    for r in results:
        if "h2" not in r:
            continue
        d, rc, nb, o1, o2 = r["d"], r["rc"], r["nb"], r["o1"], r["o2"]
        for j in range(r["rows"].n):
            m1 = _row_out(r["h1"], r["rows"], j)
            pix = dict(zeta=m1["zeta"], J=m1["J"], u1=m1["u1"], u2=m1["u2"], seff=m1["seff"])
            ref = OK.pass2(d["sb"][j], G.row_dict(rc, j), G.nb_row(nb, j), r["odet"], d["s0"], d["axis"],
                           d["frames_phi0"], d["osc"], d["p2_sd"], d["p2_sm"], d["p2_gain"], d["prof"], m1["bg"],
                           m1["nbg"], d["p2_rcw"], pix)
            mine = {k: r["h2"][k][j] for k in r["h2"]}
            ctx_o = dict(ref, vsum=m1["vsum"])
            for k in ref:
                ok, worst = T.within(k, mine[k], ref[k], ctx_o, rel=2e-6)
                assert ok, ("oracle", case, r["chunk"], j, k, worst, mine[k], ref[k])
            ctx = {k: o2[k][j] for k in o2}
            for k in ("iprf", "vprf", "vprf0", "corr", "p_valid", "p_total", "ipartner", "rho", "p_fg"):
                ok, worst = T.within(k, mine[k], o2[k][j], ctx)
                assert ok, ("reference", case, r["chunk"], j, k, worst, mine[k], o2[k][j])
            n += 1
    assert n > 0 or case == "sigmas"


def test_accumulate_and_finalize_match_oracle():
    """Profile accumulation of every stored pass-1 chunk's strong rows (float64 grids) and the finalised
    profiles."""
    from xpg_b200 import device as D
    case = "adaptive"
    spec, tmpl, mask, excl = G.case_inputs(case)
    g = spec.geometry()
    det = D.DeviceDetector(g, tmpl)
    nreg = spec.n_regions_xy ** 2
    num_o = np.zeros((nreg, 41, 41))
    den_o = np.zeros((nreg, 41, 41))
    num = torch.zeros((nreg, 41, 41), dtype=torch.float64, device="cuda")
    den = torch.zeros_like(num)
    n_strong = 0
    for i in G.chunks(case):
        d, rc, nb, o1, o2 = G.chunk(case, i)
        rows = _rows_from_chunk(d, rc, nb, "cuda")
        arena = torch.as_tensor(d["sb"].reshape(-1)).cuda()
        blk, keep = _block(d)
        p1 = D.Pass1Buffers(rows)
        D.pass1(det, rows, blk, arena, p1)
        D.accumulate(rows, p1, nreg, num, den)
        h1 = {k: v.cpu().numpy() for k, v in p1.t.items()}
        for j in range(rows.n):
            o = _row_out(h1, rows, j)
            if OK.is_strong_for_profiles(o):
                OK.accumulate(num_o, den_o, o, int(rc["region"][j]))
                n_strong += 1
    assert n_strong > 10
    np.testing.assert_allclose(num.cpu().numpy(), num_o, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(den.cpu().numpy(), den_o, rtol=1e-12, atol=1e-12)
    prof = torch.empty((nreg, 41, 41), dtype=torch.float32, device="cuda")
    D.finalize_profiles(num, den, prof)
    want = OK.finalize_profiles(num_o, den_o)
    got = prof.cpu().numpy()
    assert np.max(np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), 1e-30)) < 2.5e-7


@pytest.mark.parametrize("with_partner", [False, True])
def test_largest_box_matches_oracle(with_partner):
    """The largest shoebox XPG plans (97 x 97 px, 65 frames: max(XY_BUCKETS), max(DZ_BUCKETS)) through pass 1 and
    pass 2: a stored reflection's box pasted into a 97 x 97 x 65 box of Poisson background (with masked, unrecorded
    and overloaded voxels), its origin moved so that the reflection stays centred, against the oracle."""
    from xpg_b200 import device as D
    case = "crowded" if with_partner else "config1"        # a partner (joint fit) in the crowded sweep's chunks
    spec, tmpl, mask, excl = G.case_inputs(case)
    g = spec.geometry()
    det = D.DeviceDetector(g, tmpl)
    odet = OK.detector_consts(g, tmpl)
    i = next(k for k in G.chunks(case) if G.chunk(case, k)[4])
    d, rc, nb, o1, o2 = G.chunk(case, i)
    j = int(np.argmax(rc["has_p"])) if with_partner else int(np.argmin(rc["has_p"]))
    assert (rc["has_p"][j] > 0.5) == with_partner
    _, Dz0, Dy0, Dx0 = d["sb"].shape
    bx, Dz = 97, 65
    oy, ox = (bx - Dy0) // 2, (bx - Dx0) // 2
    rng = np.random.default_rng(5)
    sb = rng.poisson(1.5, (1, Dz, bx, bx)).astype(np.float32)
    sb[0, :Dz0, oy:oy + Dy0, ox:ox + Dx0] = d["sb"][j]
    flat = sb.reshape(-1)
    flat[rng.choice(flat.size, 300, replace=False)] = -1.0
    flat[rng.choice(flat.size, 30, replace=False)] = -2.0
    sb[0, :, :3, :] = -3.0                                     # unrecorded rows at the box edge
    one = {k: np.asarray(v[j:j + 1]).copy() for k, v in rc.items()}
    one["ix0"] = one["ix0"] - ox
    one["iy0"] = one["iy0"] - oy
    nb1 = {k: np.asarray(v[j:j + 1]) for k, v in nb.items()}
    rows = D.RowSet(S=one["S"], phi=one["phi"], ix0=one["ix0"], iy0=one["iy0"], iz0=one["iz0"], fb=one["fb"],
                    region=one["region"], has_p=one["has_p"], pS=one["pS"], pphi=one["pphi"],
                    pxs=np.ones(1, np.int32), Dz=np.full(1, Dz), bx=np.full(1, bx), nb=nb1, device="cuda",
                    sb_bias=0.0)
    arena = torch.as_tensor(sb.reshape(-1)).cuda()
    blk, keep = _block(d)
    p1 = D.Pass1Buffers(rows)
    D.pass1(det, rows, blk, arena, p1)
    D.status()
    h1 = {k: v.cpu().numpy() for k, v in p1.t.items()}
    mine = _row_out(h1, rows, 0)
    r0 = G.row_dict(one, 0)
    ref = OK.pass1(sb[0], r0, G.nb_row(nb1, 0), odet, d["s0"], d["axis"], d["frames_phi0"], d["osc"], d["sd"],
                   d["sm"], d["gain"], d["rcw"])
    for k in EXACT:
        assert np.array_equal(np.asarray(mine[k]).astype(np.float64), np.asarray(ref[k]).astype(np.float64)), k
    for k in ("isum", "vsum", "vsum0", "xo", "yo", "zo", "m_d", "m_m", "frac_rec", "img2", "fz"):
        ok, worst = T.within(k, mine[k], ref[k], ref, rel=1e-5)
        assert ok, (k, worst)
    prof = torch.as_tensor(d["prof"]).cuda()
    blk2, keep2 = _block(d, "p2_")
    p2 = D.Pass2Buffers(rows)
    D.pass2(det, rows, blk2, arena, prof, p1, p2)
    D.status()
    got = {k: v.cpu().numpy()[0] for k, v in p2.t.items()}
    pix = dict(zeta=mine["zeta"], J=mine["J"], u1=mine["u1"], u2=mine["u2"], seff=mine["seff"])
    want = OK.pass2(sb[0], r0, G.nb_row(nb1, 0), odet, d["s0"], d["axis"], d["frames_phi0"], d["osc"], d["p2_sd"],
                    d["p2_sm"], d["p2_gain"], d["prof"], mine["bg"], mine["nbg"], d["p2_rcw"], pix)
    ctx = dict(want, vsum=mine["vsum"])
    for k in want:
        ok, worst = T.within(k, got[k], want[k], ctx, rel=2e-6)
        assert ok, (k, worst, got[k], want[k])


def test_batched_passes_match_per_shape_launches():
    """Pass 1 and pass 2 of the stored chunks of every fixture (several detectors, block constants, box shapes and
    neighbour column counts) in shared persistent launches (xi_pass1_batched / xi_pass2_batched, size bins of the
    box side) give the same bits as one launch per shape (xi_pass1 / xi_pass2)."""
    from xpg_b200 import device as D
    sets, ref, keep = [], [], []
    for case in CASES:
        spec, tmpl, mask, excl = G.case_inputs(case)
        det = D.DeviceDetector(spec.geometry(), tmpl)
        for i in G.chunks(case):
            d, rc, nb, o1, o2 = G.chunk(case, i)
            if not o2:
                continue
            rows = _rows_from_chunk(d, rc, nb, "cuda")
            arena = torch.as_tensor(d["sb"].reshape(-1)).cuda()
            blk, k1 = _block(d)
            blk2, k2 = _block(d, "p2_")
            prof = torch.as_tensor(d["prof"]).cuda()
            a1, a2 = D.Pass1Buffers(rows), D.Pass2Buffers(rows)          # one launch per shape
            D.pass1(det, rows, blk, arena, a1)
            D.pass2(det, rows, blk2, arena, prof, a1, a2)
            b1, b2 = D.Pass1Buffers(rows), D.Pass2Buffers(rows)          # batched
            sets.append((D.rowset_entry(det, rows, blk, arena, b1), D.rowset_entry(det, rows, blk2, arena, b1, prof,
                                                                                   b2)))
            ref.append((a1, a2, b1, b2, rows))
            keep += [det, arena, k1, k2, prof]
    D.status()
    n = len(sets)
    groups = [(s, np.arange(r[4].n), r[4].bx, r[4].Dz) for s, r in enumerate(ref)]
    t1 = D.RowSetTable([s[0] for s in sets])
    t2 = D.RowSetTable([s[1] for s in sets])
    for bins in ((97,), (17, 23, 41, 97)):
        launches = D.batched_items(groups, bins)
        D.pass1_batched(t1, launches)
        D.pass2_batched(t2, launches)
        D.status()
        same = lambda a, b: torch.equal(a.nan_to_num(7.0), b.nan_to_num(7.0)) if a.is_floating_point() else \
            torch.equal(a, b)
        for a1, a2, b1, b2, rows in ref:
            for k in a1.t:
                assert same(a1.t[k], b1.t[k]), (n, bins, k)
            for k in a2.t:
                assert same(a2.t[k], b2.t[k]), (n, bins, k)


def test_zero_rows_clears_only_the_listed_slots():
    """xi_zero_rows: the listed rows' slots (Dz * bx^2 floats rounded up to 4) read 0, every other float keeps its
    value."""
    import ctypes as C

    import torch
    from xpg_b200 import native as N
    Dz = np.array([2, 3, 1, 4], np.int32)
    bx = np.array([3, 2, 5, 1], np.int32)
    slot = (Dz.astype(np.int64) * bx * bx + 3) // 4 * 4
    off = np.concatenate([[0], np.cumsum(slot)[:-1]]).astype(np.int64)
    arena = torch.full((int(slot.sum()) + 4,), 7.0, dtype=torch.float32, device="cuda")
    t = {k: torch.from_numpy(v).cuda() for k, v in dict(Dz=Dz, bx=bx, sb_off=off).items()}
    order = torch.tensor([1, 3], dtype=torch.int32, device="cuda")
    g = N.XiGatherRows()
    g.n = 4
    g.Dz, g.bx, g.sb_off = N.ptr(t["Dz"]), N.ptr(t["bx"]), N.ptr(t["sb_off"])
    g.order, g.n_order = N.ptr(order), 2
    N.check(N.load().xi_zero_rows(C.byref(g), N.ptr(arena), N.stream_handle()), "xi_zero_rows")
    a = arena.cpu().numpy()
    want = np.full(a.size, 7.0, np.float32)
    for r in (1, 3):
        want[off[r]:off[r] + slot[r]] = 0.0
    np.testing.assert_array_equal(a, want)
