"""The library's host Bitshuffle/LZ4 encoder (dg_bslz4_compress) on the CPU:
its chunks decode with the oracle to the original frame, carry the header
the format defines, stay within dg_bslz4_bound, and invalid arguments are
rejected. No device is needed."""
import struct

import numpy as np
import pytest


@pytest.fixture(scope="module")
def dg():
    from dioptrin_b200 import build
    build.build()
    import dioptrin_b200 as d
    return d


FRAMES = [((65, 67), 0), ((65, 67), 1024), ((300, 201), 2048), ((7, 3), 0), ((1, 5), 0),
          ((128, 64), 8192), ((50, 50), 49152), ((33, 40), 32)]


@pytest.mark.parametrize("dtype", [np.uint16, np.uint32, np.int32])
@pytest.mark.parametrize("shape,block", FRAMES)
def test_chunks_decode_to_the_frame(dg, oracle, dtype, shape, block):
    rng = np.random.default_rng(hash((shape, block)) % 2**32)
    f = rng.poisson(3.0, shape).astype(dtype)
    f.flat[:5] = np.iinfo(dtype).max // 3
    if np.dtype(dtype) == np.int32:
        f.flat[5:9] = -7  # negative pixels (detector gaps) are bit patterns too
    c = dg.bslz4_compress(f, block)
    total, hdr_block = struct.unpack(">QI", c[:12])
    assert total == f.nbytes and hdr_block == block
    assert len(c) <= dg._native.lib().dg_bslz4_bound(f.size, f.itemsize, block)
    assert np.array_equal(oracle.bslz4_decode(c, dtype, f.size).reshape(shape), f)


def test_compressible_frames_compress(dg):
    f = np.zeros((512, 512), np.uint32)
    f[::7, ::5] = 3
    c = dg.bslz4_compress(f)
    assert len(c) < f.nbytes / 20


def test_invalid_arguments(dg):
    with pytest.raises(TypeError):
        dg.bslz4_compress(np.zeros(16, np.float32))
    for block in (12, 8 * 4 + 4, 64 * 1024):
        with pytest.raises(ValueError):
            dg.bslz4_compress(np.zeros(64, np.uint32), block)
    assert dg._native.lib().dg_bslz4_bound(10, 3, 0) == -1
