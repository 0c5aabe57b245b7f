"""Oracle of the bitshuffle-LZ4 frame decode (HDF5 filter 32008, Eiger chunks): TEST INFRASTRUCTURE (see
oracle/__init__.py).

References: the chunk layout and the LZ4 stage `xpg/io/bslz4.py:1-10`, `:35-64` (`lz4_stage`); the bit unshuffle
`xpg/io/bslz4.py:28-32` (`_bitunshuffle`) and `:85-121` (`unshuffle_frame_torch`: full blocks, then the last
partial block's multiple of 8 elements shuffled as one block, then its n % 8 elements stored as they are). XPG takes
the LZ4 block decompression from the `lz4` package (`lz4.block.decompress`, absent here); it is restated from the
published LZ4 block format: sequences of a token (literal length in the high nibble, match length - 4 in the low
nibble, 15 meaning "more length bytes follow, each added, until one below 255"), the literals, then a 2-byte
little-endian match offset and the match length's extra bytes; the last sequence has literals only; a match may
overlap its own output (offset < length: byte by byte).

Not pinned by reference outputs (the reference needs lz4 / h5py / hdf5plugin, absent here): pinned by known-answer
LZ4 blocks written by hand from the format, and by round trips through the encoder below, which exists only to make
test chunks (greedy LZ4 matching; standard end-of-block rules: the last 5 bytes are literals and no match starts in
the last 12).
"""
from __future__ import annotations

import numpy as np

DEFAULT_BLOCK_BYTES = 8192


# ---- LZ4 block format ---------------------------------------------------------------------------------------------
def lz4_decompress(src, n_out):
    """LZ4 block -> n_out bytes (ValueError on a malformed block)."""
    src = bytes(src)
    out = bytearray()
    ip, n = 0, len(src)
    while True:
        if ip >= n:
            raise ValueError("lz4: truncated block")
        token = src[ip]
        ip += 1
        lit = token >> 4
        if lit == 15:
            while True:
                if ip >= n:
                    raise ValueError("lz4: truncated literal length")
                b = src[ip]
                ip += 1
                lit += b
                if b != 255:
                    break
        if ip + lit > n:
            raise ValueError("lz4: literals beyond the block")
        out += src[ip:ip + lit]
        ip += lit
        if ip == n:                        # the last sequence: literals only
            break
        if ip + 2 > n:
            raise ValueError("lz4: truncated offset")
        off = src[ip] | (src[ip + 1] << 8)
        ip += 2
        ml = token & 15
        if ml == 15:
            while True:
                if ip >= n:
                    raise ValueError("lz4: truncated match length")
                b = src[ip]
                ip += 1
                ml += b
                if b != 255:
                    break
        ml += 4
        if off == 0 or off > len(out):
            raise ValueError("lz4: match offset outside the output")
        start = len(out) - off
        for k in range(ml):                # overlapping copies repeat the pattern
            out.append(out[start + k])
        if len(out) > n_out:
            raise ValueError("lz4: output beyond its size")
    if len(out) != n_out:
        raise ValueError("lz4: output size differs")
    return bytes(out)


def _lz4_len(v):
    out = bytearray()
    while v >= 255:
        out.append(255)
        v -= 255
    out.append(v)
    return out


def lz4_compress(data):
    """A valid LZ4 block of data (greedy matching of 4-byte prefixes; test chunks only)."""
    data = bytes(data)
    n = len(data)
    out = bytearray()
    table = {}
    anchor = ip = 0
    mflimit = n - 12
    while ip < mflimit:
        key = data[ip:ip + 4]
        cand = table.get(key)
        table[key] = ip
        if cand is None or ip - cand > 65535:
            ip += 1
            continue
        ml = 4
        while ip + ml < n - 5 and data[cand + ml] == data[ip + ml]:
            ml += 1
        lit = ip - anchor
        token = (min(lit, 15) << 4) | min(ml - 4, 15)
        out.append(token)
        if lit >= 15:
            out += _lz4_len(lit - 15)
        out += data[anchor:ip]
        off = ip - cand
        out += bytes((off & 255, off >> 8))
        if ml - 4 >= 15:
            out += _lz4_len(ml - 4 - 15)
        ip += ml
        anchor = ip
    lit = n - anchor
    out.append(min(lit, 15) << 4)
    if lit >= 15:
        out += _lz4_len(lit - 15)
    out += data[anchor:]
    return bytes(out)


# ---- bit shuffle --------------------------------------------------------------------------------------------------
def bitunshuffle(buf, n, esize):
    """n elements (n a multiple of 8) of esize bytes from their bit planes: plane 8 b + k holds bit k of byte b of
    every element, element j at bit j % 8 of byte j // 8 (`xpg/io/bslz4.py:28-32`)."""
    bits = np.unpackbits(np.frombuffer(bytes(buf), np.uint8).reshape(8 * esize, n // 8), axis=1, bitorder="little")
    return np.packbits(bits.T, axis=1, bitorder="little").reshape(-1)


def bitshuffle(elem_bytes, n, esize):
    """Inverse of bitunshuffle (test chunks only)."""
    bits = np.unpackbits(np.frombuffer(bytes(elem_bytes), np.uint8).reshape(n, esize), axis=1, bitorder="little")
    return np.packbits(bits.T, axis=1, bitorder="little").reshape(-1)


# ---- chunks -------------------------------------------------------------------------------------------------------
def _block_elems(block_bytes, esize):
    b = (block_bytes or DEFAULT_BLOCK_BYTES) // esize
    return b - b % 8


def encode_chunk(values, esize, block_bytes=DEFAULT_BLOCK_BYTES):
    """bitshuffle-LZ4 chunk of a frame's values (uint32 or uint16): 8-byte big-endian size, 4-byte big-endian block
    size, then per block a 4-byte big-endian compressed size and the LZ4 block; a last partial block's n % 8
    elements follow as they are."""
    v = np.ascontiguousarray(values).reshape(-1)
    raw = v.astype(np.uint32 if esize == 4 else np.uint16).view(np.uint8)
    n = v.size
    belem = _block_elems(block_bytes, esize)
    out = bytearray((n * esize).to_bytes(8, "big") + int(block_bytes).to_bytes(4, "big"))
    done = 0
    while done < n:
        m = min(belem, n - done)
        m8 = m - m % 8
        if m8:
            sh = bitshuffle(raw[done * esize:(done + m8) * esize], m8, esize)
            c = lz4_compress(sh.tobytes())
            out += len(c).to_bytes(4, "big") + c
        if m8 < m:
            out += raw[(done + m8) * esize:(done + m) * esize].tobytes()
        done += m
    return bytes(out)


def lz4_stage(chunk, esize):
    """The chunk's blocks LZ4-decompressed, still bit-shuffled (`xpg/io/bslz4.py:35-64`): (bytes, block elements)."""
    mv = memoryview(bytes(chunk))
    total = int.from_bytes(mv[0:8], "big")
    block = int.from_bytes(mv[8:12], "big")
    if total % esize:
        raise ValueError("not a chunk of this element size")
    n = total // esize
    belem = _block_elems(block, esize)
    out = bytearray()
    pos, done = 12, 0
    while done < n:
        m = min(belem, n - done)
        m8 = m - m % 8
        if m8:
            c = int.from_bytes(mv[pos:pos + 4], "big")
            pos += 4
            out += lz4_decompress(mv[pos:pos + c], m8 * esize)
            pos += c
        if m8 < m:
            out += mv[pos:pos + (m - m8) * esize]
            pos += (m - m8) * esize
        done += m
    return bytes(out), belem


def unshuffle(buf, n, esize, belem):
    """Element bytes of a frame from its LZ4-stage output (`xpg/io/bslz4.py:85-107`)."""
    buf = np.frombuffer(bytes(buf), np.uint8)
    out = np.empty(n * esize, np.uint8)
    nf = n // belem
    for k in range(nf):
        a = k * belem * esize
        out[a:a + belem * esize] = bitunshuffle(buf[a:a + belem * esize], belem, esize)
    a = nf * belem * esize
    rem = n - nf * belem
    r8 = rem - rem % 8
    if r8:
        out[a:a + r8 * esize] = bitunshuffle(buf[a:a + r8 * esize], r8, esize)
    out[a + r8 * esize:] = buf[a + r8 * esize:n * esize]
    return out


def decode_chunk(chunk, n, esize):
    """uint32 frame values of a chunk; uint16 counts widened with their all-ones value (saturated / masked) mapped
    to 0xFFFFFFFF, the flag the uint32 frame path reads (`xpg/io/bslz4.py:114-116`: 2^n - 1 -> masked)."""
    buf, belem = lz4_stage(chunk, esize)
    b = unshuffle(buf, n, esize, belem)
    if esize == 4:
        return b.view(np.uint32).copy()
    v = b.view(np.uint16).astype(np.uint32)
    v[v == 0xFFFF] = 0xFFFFFFFF
    return v
