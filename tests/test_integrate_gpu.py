"""End-to-end GPU parity of the drop-in `integrate()` / `estimate_sigmas()` against the reference's own results on
the golden sweeps (frames re-rendered from the fixture's seed and checked by crc)."""
from __future__ import annotations

import json

import numpy as np
import pytest

import golden_io as G
import tolerance as T

pytestmark = pytest.mark.gpu

EXACT_INT = ("n_over", "n_fg_masked", "iz0", "dz", "fb", "region", "ix0", "iy0", "overlap", "hkl", "block", "lattice")
CHECK_F = ("bg", "isum", "vsum", "vsum0", "iprf", "vprf", "vprf0", "xo", "yo", "zo", "frac_rec", "m_d", "m_m",
           "corr", "p_valid", "p_total", "rho", "p_fg")


def _run(case, images=None, **over):
    from xpg_b200 import frames as FR
    from xpg_b200.integrate import integrate
    from xpg_b200.plan import IntegrationModel
    z = G.load(case)
    spec, tmpl, mask, excl = G.case_inputs(case)
    exp = spec.experiment()
    edges = z["edges"]
    if images is None:
        images = FR.U32Frames(G.frames_of(case), first=1, overload=spec.overload)
    model = IntegrationModel(sigma_d=spec.sigma_d, sigma_m=spec.sigma_m, gain=1.0)
    kw = dict(frames=(1, spec.nframes), mask=mask, minimum_zeta=0.05, verbose=False,
              n_regions_xy=spec.n_regions_xy, exclude_frames=excl, bkg_template=tmpl,
              foreign_spots=G.foreign_of(case))
    kw.update(over)
    return integrate(images, [exp] * (len(edges) - 1), edges, model, float(z["dmin"]), **kw)


def _compare(case, res):
    z = G.load(case)
    out = {k[4:]: v for k, v in z.items() if k.startswith("out_")}
    r = res.refl
    assert len(r["x"]) == len(out["x"])
    for k in EXACT_INT:
        assert np.array_equal(np.asarray(r[k]), np.asarray(out[k])), (case, k)
    worst = {}
    for k in CHECK_F:
        mine, ref = np.asarray(r[k], np.float64), np.asarray(out[k], np.float64)
        bad = []
        for j in range(len(ref)):
            ctx = {kk: out[kk][j] for kk in ("isum", "vsum", "vprf", "p_valid", "p_total", "m_m")}
            ctx["seff"] = 1e-3
            ok, w = T.within(k, mine[j], ref[j], ctx)
            worst[k] = max(worst.get(k, 0.0), w)
            if not ok:
                bad.append((j, mine[j], ref[j]))
        assert not bad, (case, k, len(bad), bad[:3])
    return worst


@pytest.mark.parametrize("case", G.CASES)
def test_integrate_matches_reference(case):
    res = _run(case)
    z = G.load(case)
    # per-block adapted widths (they feed pass 2)
    bp = json.loads(str(z["bp_json"]))
    for b, v in bp.items():
        mine = res.block_params[int(b)]
        assert mine["n"] == v["n"], (b, mine, v)
        assert abs(mine["sigma_m"] - v["sigma_m"]) <= 1e-6 * v["sigma_m"], (b, mine, v)
        assert abs(mine["sigma_d"] - v["sigma_d"]) <= 1e-6 * v["sigma_d"], (b, mine, v)
        assert np.allclose(mine["rcw"], v["rcw"], atol=1.5e-3), (b, mine, v)
    # learnt profiles of every block
    for k in z:
        if k.startswith("prof_"):
            b = int(k[5:])
            for reg in range(z[k].shape[0]):
                peak = float(np.abs(z[k][reg]).max())
                np.testing.assert_allclose(res.profiles[b][reg], z[k][reg], rtol=1e-5, atol=1e-5 * peak)
    worst = _compare(case, res)
    assert worst["iprf"] < T.REL


def test_imageset_float_path_identical():
    """Frames handed over as an XPG-style float32 ImageSet give bit-identical results to the raw uint32 path."""
    from xpg_b200 import frames as FR
    from xpg_b200.synth import encode_frame
    case = "binned"
    spec, tmpl, mask, excl = G.case_inputs(case)
    raw = G.frames_of(case)

    class Images:
        first, last, nx, ny = 1, spec.nframes, spec.nx, spec.ny

        def get(self, f):
            return encode_frame(raw[f - 1], spec.overload)
    a = _run(case).refl
    b = _run(case, images=FR.ImageSetFrames(Images())).refl
    for k in CHECK_F + ("n_over", "n_fg_masked"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]), equal_nan=True), k


def test_results_independent_of_wedge_size():
    """Wedge size (frames per upload and gather launch) changes nothing."""
    a = _run("binned", wedge_frames=7).refl
    b = _run("binned", wedge_frames=64).refl
    for k in CHECK_F:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]), equal_nan=True), k


@pytest.mark.parametrize("case", ["binned", "adaptive"])
def test_results_independent_of_schedule(case, monkeypatch):
    """Pass 1 of completed rows between wedge uploads (forced for every wedge), resident frames gathered in one
    wedge, and pinned host frames streamed by the transfer thread give the same results as the default schedule;
    "adaptive" has two blocks whose widths carry over."""
    import sys

    import torch
    from xpg_b200 import frames as FR
    I = sys.modules["xpg_b200.integrate"]              # the module (the package exports the function of that name)
    spec = G.case_inputs(case)[0]
    a = _run(case).refl
    resident = FR.U32Frames(torch.as_tensor(G.frames_of(case).view(np.int32)).cuda(), first=1, overload=spec.overload)
    b = _run(case, images=resident).refl
    pinned = torch.as_tensor(G.frames_of(case).view(np.int32)).pin_memory()
    d = _run(case, images=FR.U32Frames(pinned, first=1, overload=spec.overload), wedge_frames=4).refl
    monkeypatch.setattr(I, "EARLY_PASS1_ROWS", 1)
    c = _run(case, wedge_frames=3).refl
    e = _run(case, images=FR.U32Frames(pinned, first=1, overload=spec.overload), wedge_frames=3).refl
    for k in CHECK_F + ("n_over", "n_fg_masked"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]), equal_nan=True), ("resident", k)
        assert np.array_equal(np.asarray(a[k]), np.asarray(c[k]), equal_nan=True), ("early pass 1", k)
        assert np.array_equal(np.asarray(a[k]), np.asarray(d[k]), equal_nan=True), ("transfer thread", k)
        assert np.array_equal(np.asarray(a[k]), np.asarray(e[k]), equal_nan=True), ("thread + early pass 1", k)


@pytest.mark.parametrize("mode", ["packed", "exceptions_overflow"])
def test_packed_transfer_identical(mode, monkeypatch):
    """Frames uploaded packed to one byte a pixel (xi_pack_u8 on the host, xi_unpack_u8 on the device) give the
    results of the same frames resident in device memory, bit for bit: with counts planted at and around the byte
    codes' limits (253-256, 2^16, the overload threshold, 0xFFFFFFFE, flagged), and with a chunk holding more
    exception pixels than the exception list takes (that chunk is sent raw)."""
    import torch
    from xpg_b200 import frames as FR
    case = "binned"
    spec = G.case_inputs(case)[0]
    raw = G.frames_of(case).copy()
    rng = np.random.default_rng(7)
    n_f, ny, nx = raw.shape
    fixed = np.array([253, 254, 255, 256, 1 << 16, spec.overload - 1, spec.overload, 0xFFFFFFFE, 0xFFFFFFFF],
                     np.uint32)
    for f in range(n_f):
        iy, ix = rng.integers(0, ny, 40), rng.integers(0, nx, 40)
        raw[f, iy, ix] = np.where(raw[f, iy, ix] == 0xFFFFFFFF, raw[f, iy, ix], rng.choice(fixed, 40))
    if mode == "exceptions_overflow":
        iy, ix = rng.integers(0, ny, 4000), rng.integers(0, nx, 4000)
        raw[1, iy, ix] = np.where(raw[1, iy, ix] == 0xFFFFFFFF, raw[1, iy, ix], 300)
        monkeypatch.setattr(FR, "PACK_EXC_PER_PIXEL", 0.0)       # the list takes 1024 pairs per chunk
    resident = FR.U32Frames(torch.as_tensor(raw.view(np.int32)).cuda(), first=1, overload=spec.overload)
    a = _run(case, images=resident).refl
    pinned = torch.as_tensor(raw.view(np.int32)).pin_memory()
    src = FR.U32Frames(pinned, first=1, overload=spec.overload)
    b = _run(case, images=src, wedge_frames=5).refl                # both transfer threads
    assert src.transfer["chunks_packed"] > 0
    monkeypatch.setattr(FR, "RAW_THREAD", False)                  # pack every chunk the exception list allows
    only = FR.U32Frames(pinned, first=1, overload=spec.overload)
    c = _run(case, images=only, wedge_frames=5).refl
    n_chunks = only.transfer["chunks_packed"] + only.transfer["chunks_raw"]
    if mode == "exceptions_overflow":
        assert only.transfer["chunks_raw"] == 1 and only.transfer["chunks_packed"] == n_chunks - 1
    else:
        assert only.transfer["chunks_raw"] == 0 and n_chunks > 0
    for k in CHECK_F + ("n_over", "n_fg_masked"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]), equal_nan=True), (mode, "two threads", k)
        assert np.array_equal(np.asarray(a[k]), np.asarray(c[k]), equal_nan=True), (mode, "packed", k)


def test_estimate_sigmas_matches_reference():
    from xpg_b200 import frames as FR
    from xpg_b200.integrate import estimate_sigmas
    from xpg_b200.plan import IntegrationModel
    case = "sigmas"
    z = G.load(case)
    spec = G.spec_of(case)
    images = FR.U32Frames(G.frames_of(case), first=1, overload=spec.overload)
    model = estimate_sigmas(images, spec.experiment(), IntegrationModel(spec.sigma_d, spec.sigma_m),
                            max(float(z["dmin"]), 2.0), (1, spec.nframes), verbose=False)
    np.testing.assert_allclose([model.sigma_d, model.sigma_m], z["model"], rtol=1e-6)
    hist = np.array(model.history)
    assert hist.shape == z["history"].shape
    np.testing.assert_allclose(hist[:, :2], z["history"][:, :2], rtol=1e-6)
    assert np.array_equal(hist[:, 2], z["history"][:, 2])


@pytest.mark.parametrize("where", ["host", "device"])
def test_packed_store_identical(where):
    """Frames held in the packed transfer encoding (a PackedStore in pinned host memory, or resident in HBM) and
    widened wedge by wedge give bit-identical results to the same frames given raw; "binned" has excluded frames
    (never unpacked) and counts above the packed byte's range."""
    import torch
    from xpg_b200 import frames as FR
    case = "binned"
    spec = G.case_inputs(case)[0]
    raw = G.frames_of(case)
    store = FR.PackedStore(raw.shape[0], spec.ny, spec.nx)
    store.add_wedge(0, torch.from_numpy(np.ascontiguousarray(raw).view(np.int32)).pin_memory())
    assert store.index[:, 2].sum() > 0                       # exception pairs were needed
    src = FR.PackedFrames(store if where == "host" else store.to("cuda"), first=1, overload=spec.overload)
    a = _run(case).refl
    b = _run(case, images=src).refl
    for k in CHECK_F + ("n_over", "n_fg_masked", "isum_raw"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]), equal_nan=True), k
    if where == "host":
        assert src.transfer["h2d_bytes"] > 0


def test_pack_generated_frames_round_trip():
    """pack_generated: frames rendered on the device, packed on the host, widened back on the device bit for bit."""
    import torch
    from xpg_b200 import frames as FR
    from xpg_b200 import synth
    spec = synth.config1(nframes=12)
    _, table = synth.reflection_table(spec)
    ref = synth.device_frames(spec, table, 1, 12)
    store = FR.pack_generated(lambda k, n, out: out.copy_(ref[k:k + n]), 12, spec.ny, spec.nx, wedge=5)
    dev = store.to("cuda")
    out = torch.empty((spec.ny, spec.nx), dtype=torch.int32, device="cuda")
    for k in range(12):
        dev.unpack(k, out, torch.cuda.current_stream())
        assert torch.equal(out, ref[k]), k


def test_integration_in_parts_under_a_memory_budget():
    """A device budget below the open blocks' buffers: each phi block is integrated in parts of consecutive phi
    (own profiles and widths), as XPG does when its host budget is short (its own test of split integration,
    tests/test_pipeline.py:146-177, asks for the same reflections and a small median |dI| / sigma). Here the
    100-frame sweep's single block goes in parts (with passes over the frames where the parts overlap), each with
    the widths adapted by the parts before it and the profiles learnt from its own strong spots: summation
    intensities move by a small fraction of sigma (median < 0.1), profile-fitted ones by more (median < 0.35)."""
    from xpg_b200 import memplan
    from xpg_b200.plan import IntegrationModel, plan_integration
    case = "config1"
    z = G.load(case)
    spec = G.case_inputs(case)[0]
    edges = z["edges"]
    p = plan_integration([spec.experiment()] * (len(edges) - 1), edges, IntegrationModel(spec.sigma_d, spec.sigma_m),
                         float(z["dmin"]), 1e9, (1, spec.nframes), 0.05, spec.n_regions_xy, True, True)
    one, _ = memplan.peak_bytes(p.blocks_refl, p.need_lo, p.need_hi, memplan.row_bytes(p), spec.nframes)
    wedges = 3 * 32 * spec.ny * spec.nx * 4
    a = _run(case).refl
    res = _run(case, mem_budget=0.92 * one + wedges)
    b = res.refl
    assert res.memory["parts"] > 1 and len(res.profiles) == res.memory["parts"]
    np.testing.assert_array_equal(a["hkl"], b["hkl"])
    ok = np.isfinite(a["iprf"]) & np.isfinite(b["iprf"]) & (a["vprf"] > 0) & (a["vsum"] > 0)
    assert ok.mean() > 0.9
    ds = np.abs(a["isum"][ok] - b["isum"][ok]) / np.sqrt(a["vsum"][ok])
    assert np.median(ds) < 0.1
    d = np.abs(a["iprf"][ok] - b["iprf"][ok]) / np.sqrt(a["vprf"][ok])
    assert np.median(d) < 0.35


@pytest.mark.parametrize("case", ["binned", "adaptive"])
@pytest.mark.parametrize("mode", [dict(graphs=True, overlap=False), dict(overlap=True), dict(graphs=True, overlap=True)])
def test_gather_graph_and_overlap_identical(case, mode):
    """Each wedge's gathers replayed from a CUDA graph (captured once per set of open blocks, the wedge's frames and
    rows in a device descriptor), and gathers on a stream of their own running ahead of the passes, give the same
    bits as direct launches on one stream; "binned" has excluded frames, "adaptive" two blocks open at once."""
    a = _run(case, wedge_frames=8, overlap=False).refl
    b = _run(case, wedge_frames=8, **mode).refl
    for k in CHECK_F + ("n_over", "n_fg_masked", "isum_raw"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]), equal_nan=True), k


def test_integration_in_passes_over_the_frames():
    """A budget below the two open blocks: the blocks go in passes over the frames (XPG's grouping of blocks m apart
    in phi); every reflection is integrated, the same reflections as one pass, profile-fitted intensities within a
    fraction of sigma."""
    from xpg_b200 import memplan
    from xpg_b200.plan import IntegrationModel, plan_integration
    case = "adaptive"
    z = G.load(case)
    spec = G.case_inputs(case)[0]
    edges = z["edges"]
    p = plan_integration([spec.experiment()] * (len(edges) - 1), edges, IntegrationModel(spec.sigma_d, spec.sigma_m),
                         float(z["dmin"]), 1e9, (1, spec.nframes), 0.05, spec.n_regions_xy, True, True)
    one, _ = memplan.peak_bytes(p.blocks_refl, p.need_lo, p.need_hi, memplan.row_bytes(p), spec.nframes)
    wedges = 3 * 32 * spec.ny * spec.nx * 4
    a = _run(case).refl
    res = _run(case, mem_budget=0.55 * one + wedges)
    b = res.refl
    assert len(res.memory.get("passes", [])) > 1
    np.testing.assert_array_equal(a["hkl"], b["hkl"])
    assert np.isfinite(b["iprf"]).sum() >= 0.99 * np.isfinite(a["iprf"]).sum()
    ok = np.isfinite(a["iprf"]) & np.isfinite(b["iprf"]) & (a["vprf"] > 0)
    d = np.abs(a["iprf"][ok] - b["iprf"][ok]) / np.sqrt(a["vprf"][ok])
    assert np.median(d) < 0.35                            # parts of a small sweep learn profiles from few spots


@pytest.mark.parametrize("case", ["adaptive", "superpix", "crowded"])
def test_reused_buffers_hold_no_stale_voxels(case):
    """Arenas come from the buffer pool without a full clear: every voxel a pass reads must have been gathered or
    cleared at block opening. With buffers kept between calls and every kept float32 buffer filled with NaN before
    the second call, the results equal a run on fresh buffers bit for bit."""
    import torch
    from xpg_b200 import device as D
    a = _run(case, wedge_frames=8).refl
    D.keep_buffers(True)
    try:
        _run(case, wedge_frames=8)
        for (_, dt), pool in D.POOL.free.items():
            for t in pool:
                if dt == torch.float32:
                    t.fill_(float("nan"))
        b = _run(case, wedge_frames=8).refl
    finally:
        D.keep_buffers(False)
    for k in CHECK_F + ("n_over", "n_fg_masked", "isum_raw"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]), equal_nan=True), k
