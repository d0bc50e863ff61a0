"""Bitshuffle/LZ4 chunk writers for the tests, restating how the reference's
own tests write chunks: src/integration/metal/tests.rs:298-356 (a
literals-only LZ4 stream) and src/integration/metal/bench.rs:150-230 (runs
encoded as offset-1 matches). Test infrastructure only."""
import struct

import numpy as np


def bitshuffle(raw: bytes, elem: int) -> bytes:
    a = np.frombuffer(raw, np.uint8).reshape(-1, elem)
    count = a.shape[0]
    bits = np.unpackbits(a, axis=1, bitorder="little")  # (count, 8*elem), bit p of element
    planes = bits.T.reshape(8 * elem, count // 8, 8)      # plane p, byte k, bit i
    return np.packbits(planes, axis=2, bitorder="little").tobytes()


def ext(n):
    out = bytearray()
    while n >= 255:
        out.append(255)
        n -= 255
    out.append(n)
    return bytes(out)


def lz4_literals(data: bytes) -> bytes:
    n = len(data)
    tok = (min(n, 15) << 4)
    return bytes([tok]) + (ext(n - 15) if n >= 15 else b"") + data


def lz4_runs(data: bytes) -> bytes:
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
                out += ext(len(lit) - 15)
            out += lit + struct.pack("<H", 1)
            if mlen - 4 >= 15:
                out += ext(mlen - 4 - 15)
            i += run
            anchor = i
        else:
            i += run
    out += lz4_literals(data[anchor:])
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
        z = lz4(bitshuffle(p, elem))
        out += struct.pack(">I", len(z)) + z
    if tail:
        out += raw[(n_full * be + rem_comp) * elem:]
    return bytes(out)
