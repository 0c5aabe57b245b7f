"""Bitshuffle-LZ4 frames (Eiger chunks, HDF5 filter 32008): the oracle against known-answer LZ4 blocks and round
trips; the library's LZ4 stage (host code, runs here without a GPU) against the oracle; on the GPU the bit unshuffle
against the oracle and integrate() from chunks against the same frames given raw. Cases follow the reference's own
test of the path (`tests/test_robustness.py:72-120`): a frame size that is neither a multiple of the block nor of 8,
saturated / overloaded counts, uint32 and uint16."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from oracle import bslz4 as B
from xpg_b200 import native


def test_lz4_known_blocks():
    assert B.lz4_decompress(b"\x50hello", 5) == b"hello"                                  # literals only
    assert B.lz4_decompress(b"\x13a\x01\x00\x50bcdef", 13) == b"a" * 8 + b"bcdef"         # overlapping match
    lit = bytes(range(256)) + bytes(range(44))
    assert B.lz4_decompress(b"\xf0" + bytes([255, 30]) + lit, 300) == lit                  # long literal run
    assert B.lz4_decompress(b"\x2fab\x02\x00" + bytes([255, 10]) + b"\x50xxxxx", 291) == b"ab" * 143 + b"xxxxx"
    for bad in (b"", b"\x50hell", b"\x13a\x05\x00\x50bcdef", b"\x13a\x01"):
        with pytest.raises(ValueError):
            B.lz4_decompress(bad, 13)


def _frame(n, seed, esize):
    rng = np.random.default_rng(seed)
    if esize == 4:
        v = rng.poisson(3.0, n).astype(np.uint32)
        v[rng.choice(n, max(n // 100, 1), replace=False)] = 0xFFFFFFFF
        v[rng.choice(n, max(n // 100, 1), replace=False)] = (1 << 20) + 7
        return v
    v = rng.integers(0, 1 << 16, n).astype(np.uint16)
    v[rng.choice(n, max(n // 100, 1), replace=False)] = 0xFFFF
    return v


@pytest.mark.parametrize("esize", [4, 2])
@pytest.mark.parametrize("n", [1, 8, 37 * 61, 5000, 3 * 4096 + 13])
def test_oracle_round_trip(n, esize):
    v = _frame(n, n, esize)
    want = v.astype(np.uint32)
    if esize == 2:
        want[v == 0xFFFF] = 0xFFFFFFFF
    assert np.array_equal(B.decode_chunk(B.encode_chunk(v, esize), n, esize), want)


def _stage(chunk, esize, out_bytes, threads=0):
    lib = native.load()
    out = np.zeros(max(out_bytes, 1), np.uint8)
    nb, be = C.c_int64(-1), C.c_int64(-1)
    c = np.frombuffer(chunk, np.uint8)
    rc = lib.xi_bslz4_lz4_stage(c.ctypes.data, c.size, esize, out.ctypes.data, out_bytes, threads, C.byref(nb),
                                C.byref(be))
    return rc, out[:max(nb.value, 0)], be.value


@pytest.mark.parametrize("esize,block", [(4, 8192), (2, 8192), (4, 0), (4, 1000), (2, 24)])
@pytest.mark.parametrize("n", [1, 37 * 61, 3 * 4096 + 13])
def test_lz4_stage_matches_oracle(n, esize, block):
    v = _frame(n, 7 * n + esize, esize)
    chunk = B.encode_chunk(v, esize, block_bytes=block)
    if block == 0:                                       # a zero block size means 8192 bytes
        chunk = B.encode_chunk(v, esize)[:8] + (0).to_bytes(4, "big") + B.encode_chunk(v, esize)[12:]
    want, belem = B.lz4_stage(chunk, esize)
    for threads in (1, 0):
        rc, got, be = _stage(chunk, esize, n * esize, threads)
        assert rc == native.XI_OK
        assert be == belem
        assert got.tobytes() == want


def test_lz4_stage_rejects_malformed_chunks():
    v = _frame(5000, 1, 4)
    chunk = B.encode_chunk(v, 4)
    assert _stage(chunk, 4, 5000 * 4)[0] == native.XI_OK
    assert _stage(chunk, 4, 4999 * 4)[0] == native.XI_E_ARG            # frame larger than the buffer
    assert _stage(chunk[:-3], 4, 5000 * 4)[0] == native.XI_E_ARG       # truncated
    assert _stage(chunk, 3, 5000 * 4)[0] == native.XI_E_ARG            # element size
    bad = bytearray(chunk)
    bad[16] ^= 0xFF                                                     # a corrupted first LZ4 block
    assert _stage(bytes(bad), 4, 5000 * 4)[0] in (native.XI_OK, native.XI_E_ARG)
    bad = bytearray(chunk)
    bad[12:16] = (10 ** 6).to_bytes(4, "big")                           # block size beyond the chunk
    assert _stage(bytes(bad), 4, 5000 * 4)[0] == native.XI_E_ARG
    assert _stage(chunk[:10], 4, 5000 * 4)[0] == native.XI_E_ARG        # shorter than the header


@pytest.mark.gpu
@pytest.mark.parametrize("esize", [4, 2])
@pytest.mark.parametrize("n,off", [(1, 0), (8, 0), (37 * 61, 0), (37 * 61, 1), (3 * 4096 + 13, 0),
                                   (4148 * 4362, 0)])
def test_bitunshuffle_matches_oracle(n, off, esize):
    import torch
    lib = native.load()
    v = _frame(n, n + esize, esize)
    want = v.astype(np.uint32)
    if esize == 2:
        want[v == 0xFFFF] = 0xFFFFFFFF
    # the LZ4 stage output: full blocks of 8192 bytes shuffled, the last partial block's multiple of 8 shuffled as one
    # block, its n % 8 elements as they are
    raw = v.view(np.uint8)
    belem = 8192 // esize
    parts, done = [], 0
    while done < n:
        m = min(belem, n - done)
        m8 = m - m % 8
        if m8:
            parts.append(B.bitshuffle(raw[done * esize:(done + m8) * esize], m8, esize))
        parts.append(raw[(done + m8) * esize:(done + m) * esize])
        done += m
    staged = np.concatenate(parts)
    assert np.array_equal(B.unshuffle(staged, n, esize, belem).view(np.uint16 if esize == 2 else np.uint32), v)
    d_in = torch.from_numpy(staged).cuda()
    out = torch.zeros(n + 4, dtype=torch.int32, device="cuda")
    rc = lib.xi_bitunshuffle(native.ptr(d_in), n, esize, belem, C.c_void_p(out.data_ptr() + 4 * off),
                             native.stream_handle())
    native.check(rc, "xi_bitunshuffle")
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32)[off:off + n], want)


@pytest.mark.gpu
@pytest.mark.parametrize("esize", [4, 2])
def test_integrate_from_chunks_identical(esize):
    """integrate() from bitshuffle-LZ4 chunks of the golden sweep's frames equals integrate() from the raw frames,
    bit for bit (uint16: the same counts as uint16, the flagged value all-ones)."""
    import golden_io as G
    from test_integrate_gpu import CHECK_F, _run
    from xpg_b200 import frames as FR
    case = "binned"
    spec = G.case_inputs(case)[0]
    raw = G.frames_of(case)
    if esize == 2:
        v16 = np.where(raw == 0xFFFFFFFF, 0xFFFF, np.minimum(raw, 0xFFFE)).astype(np.uint16)
        raw = np.where(v16 == 0xFFFF, 0xFFFFFFFF, v16.astype(np.uint32)).astype(np.uint32)
        chunks = [B.encode_chunk(f, 2) for f in v16]
    else:
        chunks = [B.encode_chunk(f, 4) for f in raw]
    a = _run(case, images=FR.U32Frames(raw, first=1, overload=spec.overload)).refl
    src = FR.BSLZ4Frames(chunks, raw.shape[1], raw.shape[2], esize=esize, first=1, overload=spec.overload)
    b = _run(case, images=src, wedge_frames=7).refl
    for k in CHECK_F + ("n_over", "n_fg_masked"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]), equal_nan=True), (esize, k)


def test_decode_fixture_is_the_band():
    """The chunk bench.py --decode times (tests/golden/bslz4_band.bin) decodes to the band it regenerates."""
    import sys
    from pathlib import Path
    g = Path(__file__).resolve().parent / "golden"
    sys.path.insert(0, str(g))
    import make_bslz4_band as M
    chunk = (g / "bslz4_band.bin").read_bytes()
    band = M.band()
    rc, got, be = _stage(chunk, 4, band.nbytes)
    assert rc == native.XI_OK
    assert np.array_equal(B.unshuffle(got, band.size, 4, be).view(np.uint32), band.reshape(-1))


def test_imageset_adapter_takes_bitshuffled_chunks():
    """An XPG image set whose frames are plain bitshuffle-LZ4 chunks (`bitshuffled_ok`, `read_chunk`) is read as
    chunks; one with a static pixel mask (whose encoding differs) or without chunks goes through `get`."""
    from xpg_b200 import frames as FR

    class Images:
        first, last, ny, nx = 1, 3, 37, 61
        dtype = np.dtype(np.uint32)
        overload, min_valid = 1 << 20, 0
        static_mask = None

        def bitshuffled_ok(self):
            return True

        def read_chunk(self, f):
            return B.encode_chunk(_frame(37 * 61, f, 4), 4)

        def get(self, f):
            raise AssertionError("not used")

    im = Images()
    src = FR.as_frame_source(im, device="cpu")
    assert isinstance(src, FR.BSLZ4Frames) and src.esize == 4 and src.overload == 1 << 20
    assert src._chunk(2).tobytes() == im.read_chunk(2)
    im.static_mask = np.ones((37, 61), bool)
    assert isinstance(FR.as_frame_source(im, device="cpu"), FR.BSLZ4Frames)    # an all-True mask masks nothing
    im.static_mask[3, 4] = False
    assert isinstance(FR.as_frame_source(im, device="cpu"), FR.ImageSetFrames)
    im.static_mask = None
    im.bitshuffled_ok = lambda: False
    assert isinstance(FR.as_frame_source(im, device="cpu"), FR.ImageSetFrames)


def _xpg_cases():
    z = np.load(Path(__file__).resolve().parent / "golden" / "bitunshuffle.npz")
    return [{k: z[f"c{i}_{k}"] for k in ("esize", "n", "block", "staged", "xpg_frame")}
            for i in range(len([k for k in z.files if k.endswith("_esize")]))], z


def _xpg_values(c):
    """XPG's decoded frame as the uint32 frame path holds it: flagged (-1) as all ones, counts as they are."""
    f = c["xpg_frame"]
    return np.where(f == -1.0, np.float64(0xFFFFFFFF), f).astype(np.uint32)


def test_oracle_unshuffle_matches_xpg_decoder():
    """The oracle's unshuffle (and its test encoder, the inverse) against XPG's own decoder's output on the same
    LZ4-stage bytes (fixture made by tests/golden/make_bitunshuffle_golden.py with the reference's
    unshuffle_frame_torch and _bitunshuffle)."""
    cases, z = _xpg_cases()
    for c in cases:
        esize, n, belem = int(c["esize"]), int(c["n"]), int(c["block"])
        v = B.unshuffle(c["staged"], n, esize, belem).view(np.uint16 if esize == 2 else np.uint32)
        want = _xpg_values(c)
        got = v.astype(np.uint32)
        if esize == 2:
            got[v == 0xFFFF] = 0xFFFFFFFF
        assert np.array_equal(got, want), (esize, n)
    np.testing.assert_array_equal(B.bitunshuffle(z["np_in"], 64, 4), z["np_out"])
    np.testing.assert_array_equal(B.bitshuffle(z["np_out"], 64, 4), z["np_in"])


@pytest.mark.gpu
def test_bitunshuffle_matches_xpg_decoder():
    """xi_bitunshuffle on the fixture's LZ4-stage bytes gives XPG's decoded frames (flagged pixels all ones)."""
    import torch
    lib = native.load()
    cases, _ = _xpg_cases()
    for c in cases:
        esize, n, belem = int(c["esize"]), int(c["n"]), int(c["block"])
        d_in = torch.from_numpy(np.ascontiguousarray(c["staged"])).cuda()
        out = torch.zeros(n, dtype=torch.int32, device="cuda")
        native.check(lib.xi_bitunshuffle(native.ptr(d_in), n, esize, belem, native.ptr(out), native.stream_handle()),
                     "xi_bitunshuffle")
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), _xpg_values(c)), (esize, n)
