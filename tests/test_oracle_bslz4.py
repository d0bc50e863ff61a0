"""The oracle's Bitshuffle/LZ4 decoder against chunks written the way the
reference's own tests write them (src/integration/metal/tests.rs:298-356: a
literals-only LZ4 stream; src/integration/metal/bench.rs:150-230: runs
encoded as offset-1 matches), on a 65 x 67 frame whose size leaves full,
partial and raw-tail blocks (metal/tests.rs:362-400)."""
import struct

import numpy as np
import pytest


def _bitshuffle(raw: bytes, elem: int) -> bytes:
    a = np.frombuffer(raw, np.uint8).reshape(-1, elem)
    count = a.shape[0]
    bits = np.unpackbits(a, axis=1, bitorder="little")  # (count, 8*elem), bit p of element
    planes = bits.T.reshape(8 * elem, count // 8, 8)      # plane p, byte k, bit i
    return np.packbits(planes, axis=2, bitorder="little").tobytes()


def _ext(n):
    out = bytearray()
    while n >= 255:
        out.append(255)
        n -= 255
    out.append(n)
    return bytes(out)


def _lz4_literals(data: bytes) -> bytes:
    n = len(data)
    tok = (min(n, 15) << 4)
    return bytes([tok]) + (_ext(n - 15) if n >= 15 else b"") + data


def _lz4_runs(data: bytes) -> bytes:
    # runs of >= 6 equal bytes become one literal and an offset-1 match
    out = bytearray()
    i = anchor = 0
    n = len(data)
    while i < n:
        run = 1
        while i + run < n and data[i + run] == data[i]:
            run += 1
        if run >= 6 and i + run < n:
            lit = data[anchor:i + 1]
            mlen = run - 1
            out.append((min(len(lit), 15) << 4) | min(mlen - 4, 15))
            if len(lit) >= 15:
                out += _ext(len(lit) - 15)
            out += lit + struct.pack("<H", 1)
            if mlen - 4 >= 15:
                out += _ext(mlen - 4 - 15)
            i += run
            anchor = i
        else:
            i += run
    out += _lz4_literals(data[anchor:])
    return bytes(out)


def encode(raw: bytes, elem: int, block: int, lz4) -> bytes:
    n = len(raw) // elem
    be = block // elem
    n_full, rem = divmod(n, be)
    rem_comp, tail = rem // 8 * 8, rem % 8
    out = bytearray(struct.pack(">QI", len(raw), block))
    pieces = [raw[b * block:(b + 1) * block] for b in range(n_full)]
    if rem_comp:
        pieces.append(raw[n_full * block:n_full * block + rem_comp * elem])
    for p in pieces:
        z = lz4(_bitshuffle(p, elem))
        out += struct.pack(">I", len(z)) + z
    if tail:
        out += raw[(n_full * be + rem_comp) * elem:]
    return bytes(out)


@pytest.mark.parametrize("dtype,block", [(np.uint16, 1024), (np.uint32, 2048),
                                         (np.int32, 8192), (np.uint16, 0)])
@pytest.mark.parametrize("lz4", [_lz4_literals, _lz4_runs])
def test_decode_reference_style_chunks(oracle, dtype, block, lz4):
    n = 65 * 67
    if np.dtype(dtype).itemsize == 2:
        frame = ((np.arange(n) * 73 + 11) % 65000).astype(dtype)
    else:
        frame = ((np.arange(n) * 197 + 5) % 500_000).astype(dtype)
    frame[100:400] = 7  # a long run: offset-1 matches
    raw = frame.tobytes()
    chunk = encode(raw, frame.itemsize, block or 8192, lz4)
    if block == 0:  # a zero block size in the header means 8192 bytes
        chunk = chunk[:8] + struct.pack(">I", 0) + chunk[12:]
    got = oracle.bslz4_decode(chunk, dtype, n)
    assert np.array_equal(got, frame)


def test_decode_rejects_malformed_chunks(oracle):
    frame = np.arange(1000, dtype=np.uint32)
    chunk = encode(frame.tobytes(), 4, 2048, _lz4_literals)
    with pytest.raises(ValueError):
        oracle.bslz4_decode(chunk[:-3], np.uint32, 1000)        # truncated
    with pytest.raises(ValueError):
        oracle.bslz4_decode(chunk, np.uint32, 999)              # wrong size
    bad = bytearray(chunk)
    bad[16] = 0x0F  # a match before any output
    with pytest.raises(ValueError):
        oracle.bslz4_decode(bytes(bad), np.uint32, 1000)
