"""The oracle's Bitshuffle/LZ4 decoder against chunks written the way the
reference's own tests write them (src/integration/metal/tests.rs:298-356: a
literals-only LZ4 stream; src/integration/metal/bench.rs:150-230: runs
encoded as offset-1 matches), on a 65 x 67 frame whose size leaves full,
partial and raw-tail blocks (metal/tests.rs:362-400)."""
import struct

import numpy as np
import pytest

from bslz4_chunks import encode, lz4_literals as _lz4_literals, lz4_runs as _lz4_runs


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
