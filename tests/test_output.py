"""The INTEGRATE stage's work after the path (`xpg/stage_integrate.py:408-447`) on CPU: LP / absorption correction,
row selection, the lattice split and the INTEGRATE.HKL writer, against XPG's own factors and writer run on the
reference's stored results (tests/golden/lp_output.npz, made by tests/golden/make_lp_golden.py)."""
from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np
import pytest

import golden_io as G
from xpg_b200 import output as O

GOLD = Path(__file__).resolve().parent / "golden" / "lp_output.npz"
CASES = ("config1", "adaptive", "superpix", "binned", "crowded", "precision")


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD)
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("case", CASES)
def test_lp_correction_and_hkl_match_reference(case, gold, tmp_path):
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    from make_lp_golden import split_hkl
    z = G.load(case)
    refl = {k[4:]: z[k] for k in z if k.startswith("out_")}
    spec = G.spec_of(case)
    exp = spec.experiment()
    main, extra = O.lp_correct(refl, exp.geom)
    keep = gold[f"{case}_keep"]
    assert np.array_equal(main["hkl"], refl["hkl"][keep])
    assert np.array_equal(main["rlp"], gold[f"{case}_rlp"])         # the same float64 operations: bit for bit
    assert [len(v["I"]) for _, v in sorted(extra.items())] == list(gold[f"{case}_n_extra"])
    p = tmp_path / "INTEGRATE.HKL"
    O.write_integrate_hkl(p, exp, main, (1, spec.nframes), spec.sigma_m, spec.sigma_d, "frame_?????.cbf")
    head, recs = split_hkl(p.read_text())
    assert "\n".join(head) == str(gold[f"{case}_hkl_head"])
    assert "\n".join(recs[:3]) == str(gold[f"{case}_hkl_first"])
    assert hashlib.sha256("\n".join(recs).encode()).hexdigest() == str(gold[f"{case}_hkl_sha"])


def test_lattice_split_and_selection():
    """Rows with a non-finite intensity or a sigma that is not positive leave; the rest split by lattice index."""
    spec = G.spec_of("config1")
    g = spec.geometry()
    rng = np.random.default_rng(0)
    n = 50
    S = rng.normal(size=(n, 3)) * 0.05 + np.asarray(g.s0)
    refl = dict(S=S, iprf=rng.uniform(1, 100, n), vprf=rng.uniform(1, 50, n), isum=rng.uniform(1, 100, n),
                vsum=rng.uniform(1, 50, n), p_valid=rng.uniform(0, 1, n), p_total=np.ones(n), corr=rng.uniform(0, 1, n),
                lattice=np.repeat([0, 1, 2, 0, 1], 10), hkl=np.arange(3 * n).reshape(n, 3))
    refl["iprf"][3] = np.nan
    refl["vprf"][12] = 0.0
    main, extra = O.lp_correct(refl, g)
    assert sorted(extra) == [0, 1]
    assert len(main["I"]) == 19 and len(extra[0]["I"]) == 19 and len(extra[1]["I"]) == 10
    assert np.all(np.isin(main["hkl"][:, 0] // 3, np.flatnonzero(refl["lattice"] == 0)))
    np.testing.assert_allclose(main["I"], main["iprf"] * main["rlp"])


def test_integrated_npz_round_trip(tmp_path):
    z = G.load("binned")
    refl = {k[4:]: z[k] for k in z if k.startswith("out_")}
    main, _ = O.lp_correct(refl, G.spec_of("binned").geometry())
    main["fz"] = np.zeros((len(main["I"]), 3))
    p = tmp_path / "xpg_integrated.npz"
    O.write_integrated_npz(p, main)
    back = np.load(p)
    assert "fz" not in back.files
    ref = tmp_path / "numpy.npz"
    np.savez_compressed(ref, **{k: v for k, v in main.items() if isinstance(v, np.ndarray) and k != "fz"})
    want = np.load(ref)
    assert sorted(back.files) == sorted(want.files)
    for k in want.files:                      # the same members, dtypes and values as numpy's own writer
        assert back[k].dtype == want[k].dtype and np.array_equal(back[k], want[k], equal_nan=True), k
    import zipfile
    with zipfile.ZipFile(p) as zf:
        assert zf.testzip() is None           # every member's CRC checks
