"""Bitshuffle/LZ4 frames decoded on the device and integrated
(dg_integrate_bslz4; the reference's integrate_bslz4,
src/integration/cuda.rs:554-564, and its Python batch1d_bslz4 /
batch2d_bslz4 / batch2d_bslz4_stack, src/python/cuda.rs:880-1256).

The decoded frames feed the same gather as uncompressed frames, so results
must equal dg_integrate's on the raw frames bit for bit; one case is also
checked against the CPU oracle directly. Chunks come from the library's
encoder and from writers restating the reference's own test chunks
(literals only, offset-1 runs); frame sizes leave ragged remainder blocks
and raw tails. Malformed chunks must be rejected, by the host parser or by
the decoder's error flag, and leave the plan usable."""
import struct

import numpy as np
import pytest

from bslz4_chunks import encode, lz4_literals, lz4_runs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


PONI = dict(pixel1=172e-6, pixel2=172e-6, distance=0.05, poni1=30.3 * 172e-6,
            poni2=33.7 * 172e-6, rot1=0.02, rot2=-0.01, wavelength=1e-10)


def _plan(dg, shape, n=90, method="pixel_split"):
    it = dg.Integrator.from_poni_dict(PONI, method=method, polarization_factor=0.97)
    mask = np.zeros(shape, np.uint8)
    mask[5, :] = 1
    it.set_mask(mask)
    return it.prepare_cuda1d(shape, n)


def _frames(shape, n, dtype, seed):
    rng = np.random.default_rng(seed)
    f = rng.poisson(20.0, (n,) + shape).astype(dtype)
    f[:, 3, :7] = np.iinfo(dtype).max // 5          # bright spot: high bit planes
    if np.dtype(dtype) == np.int32:
        f[:, 10, 4:9] = -1                           # gap pixels
    return f


def _same(a, b):
    for x, y in zip(a, b):
        if x is None:
            assert y is None
        else:
            assert np.array_equal(x, y, equal_nan=True)


# (shape, block bytes): 61 x 67 = 4087 pixels leaves a remainder block whose
# length is not a multiple of 32 elements and a 7-pixel raw tail; 32- and
# 16-byte blocks make every block 8 elements long.
CASES = [((61, 67), 0), ((61, 67), 1024), ((65, 67), 2048), ((61, 67), 49152)]


@pytest.mark.parametrize("dtype", [np.uint16, np.uint32, np.int32])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_bslz4_equals_raw_frames(dg, dtype, case):
    shape, block = CASES[case]
    plan = _plan(dg, shape)
    frames = _frames(shape, 5, dtype, seed=case)
    chunks = [dg.bslz4_compress(f, block) for f in frames]
    for flags in [(False, False), (True, False), (True, True)]:
        got = plan.integrate_bslz4_stack(chunks, np.dtype(dtype).name, *flags)
        want = plan.integrate_stack(frames, *flags)
        _same(got, want)
    plan.close()


@pytest.mark.parametrize("dtype,block", [(np.uint32, 32), (np.uint16, 16), (np.int32, 32)])
def test_eight_element_blocks(dg, dtype, block):
    shape = (21, 19)
    plan = _plan(dg, shape, n=30)
    frames = _frames(shape, 3, dtype, seed=9)
    chunks = [dg.bslz4_compress(f, block) for f in frames]
    _same(plan.integrate_bslz4_stack(chunks, np.dtype(dtype).name, True),
          plan.integrate_stack(frames, True))
    plan.close()


@pytest.mark.parametrize("writer", [lz4_literals, lz4_runs])
@pytest.mark.parametrize("dtype,block", [(np.uint16, 1024), (np.uint32, 8192), (np.int32, 2048)])
def test_reference_style_chunks(dg, writer, dtype, block):
    shape = (61, 67)
    plan = _plan(dg, shape)
    frames = _frames(shape, 3, dtype, seed=4)
    frames[:, 20:30, :] = 9  # long runs: offset-1 matches of every length
    chunks = [encode(f.tobytes(), f.itemsize, block, writer) for f in frames]
    _same(plan.integrate_bslz4_stack(chunks, np.dtype(dtype).name, True, True),
          plan.integrate_stack(frames, True, True))
    plan.close()


def test_against_the_oracle(dg, oracle):
    shape = (61, 67)
    plan = _plan(dg, shape)
    frames = _frames(shape, 2, np.uint32, seed=12)
    chunks = [dg.bslz4_compress(f) for f in frames]
    I, S, _ = plan.integrate_bslz4_stack(chunks, "uint32", True)
    p = oracle.poni(**PONI)
    mask = np.zeros(shape, np.uint8)
    mask[5, :] = 1
    table = oracle.compact(oracle.build_ps1d(p, *shape, 90), mask.ravel())
    norm = oracle.centres(p, *shape, polarization_factor=0.97)["norm"]
    den = oracle.denominators(table, norm)
    for k in range(len(frames)):
        sig = oracle.bslz4_decode(chunks[k], np.uint32, frames[k].size).astype(np.float64)
        yi, ys = oracle.integrate_strict(table, den, sig, True)
        fin = np.isfinite(yi)
        assert np.array_equal(fin, np.isfinite(I[k]))
        np.testing.assert_allclose(I[k][fin], yi[fin], rtol=1e-5, atol=1e-12)
        np.testing.assert_allclose(S[k][fin], ys[fin], rtol=1e-5, atol=1e-12)
    plan.close()


def test_many_batches_pinned_and_pageable(dg):
    # 150 frames run as three batches through both copy slots.
    import torch
    shape = (40, 44)
    plan = _plan(dg, shape, n=50)
    frames = _frames(shape, 150, np.uint32, seed=3)
    frames += np.arange(150, dtype=np.uint32)[:, None, None]  # every frame differs
    chunks = [dg.bslz4_compress(f) for f in frames]
    want = plan.integrate_stack(frames, True)
    _same(plan.integrate_bslz4_stack(chunks, "uint32", True), want)
    pinned = []
    for c in chunks:
        t = torch.empty(len(c), dtype=torch.uint8, pin_memory=True)
        t.numpy()[:] = np.frombuffer(c, np.uint8)
        pinned.append(t.numpy())
    _same(plan.integrate_bslz4_stack(pinned, "uint32", True), want)
    # batch1d_bslz4 results carry the radial axis
    res = plan.batch1d_bslz4(chunks[:3], "uint32", errors=True)
    assert len(res) == 3 and np.array_equal(res[2].intensity, want[0][2])
    assert np.array_equal(res[0].radial, plan.radial_array)
    assert plan.batch1d_bslz4([], "uint32") == []
    plan.close()


def test_2d_plans(dg):
    shape = (61, 67)
    it = dg.Integrator.from_poni_dict(PONI, method="pixel_split", unit="2th_deg")
    plan = it.prepare_cuda2d(shape, 40, 36)
    frames = _frames(shape, 4, np.uint16, seed=5)
    chunks = [dg.bslz4_compress(f) for f in frames]
    I, S = plan.batch2d_bslz4_stack(chunks, "uint16", errors=True)
    ri, rs, _ = plan.integrate_stack(frames, True)
    assert I.shape == (4, 36, 40)
    assert np.array_equal(I.reshape(4, -1), ri, equal_nan=True)
    assert np.array_equal(S.reshape(4, -1), rs, equal_nan=True)
    res = plan.batch2d_bslz4(chunks, "uint16")
    assert np.array_equal(res[1].intensity, ri[1], equal_nan=True)
    plan.close()


def test_malformed_chunks_are_rejected(dg):
    shape = (61, 67)
    plan = _plan(dg, shape)
    frames = _frames(shape, 2, np.uint32, seed=8)
    good = [dg.bslz4_compress(f) for f in frames]
    want = plan.integrate_stack(frames)
    with pytest.raises(ValueError, match="does not match plan frame size"):
        plan.integrate_bslz4_stack([good[0], dg.bslz4_compress(frames[0][:-1])], "uint32")
    with pytest.raises(ValueError, match="does not match plan frame size"):
        plan.integrate_bslz4_stack(good, "uint16")
    with pytest.raises(ValueError, match="truncated"):
        plan.integrate_bslz4_stack([good[0], good[1][:-40]], "uint32")
    with pytest.raises(ValueError, match="shorter than"):
        plan.integrate_bslz4_stack([good[0][:8]], "uint32")
    bad_block = good[0][:8] + struct.pack(">I", 12) + good[0][12:]
    with pytest.raises(ValueError, match="block size"):
        plan.integrate_bslz4_stack([bad_block], "uint32")
    # a match reaching before the block's start: found by the decoder
    c = bytearray(good[1])
    c[16:19] = bytes([0x0F, 0xFF, 0x7F])  # token: no literals, match at distance 0x7FFF
    with pytest.raises(ValueError, match="corrupt or truncated"):
        plan.integrate_bslz4_stack([good[0], bytes(c)], "uint32")
    with pytest.raises(TypeError):
        plan.integrate_bslz4_stack(good, "float32")
    with pytest.raises(TypeError):
        plan.integrate_bslz4_stack(good[0], "uint32")
    # the plan still integrates
    _same(plan.integrate_bslz4_stack(good, "uint32"), want)
    plan.close()


def test_corrupted_payload_never_faults(dg):
    # Random byte changes inside LZ4 payloads: each call either raises
    # ValueError or decodes some frame; the plan stays usable throughout.
    shape = (61, 67)
    plan = _plan(dg, shape)
    frames = _frames(shape, 1, np.uint32, seed=1)
    good = dg.bslz4_compress(frames[0])
    want = plan.integrate_stack(frames)
    rng = np.random.default_rng(0)
    rejected = 0
    for _ in range(40):
        c = bytearray(good)
        for pos in rng.integers(16, len(c) - 30, 4):
            c[pos] = int(rng.integers(0, 256))
        try:
            plan.integrate_bslz4_stack([bytes(c)], "uint32")
        except ValueError:
            rejected += 1
    assert rejected > 0
    _same(plan.integrate_bslz4_stack([good], "uint32"), want)
    plan.close()


def test_decode_is_timed_and_counted(dg):
    import ctypes as C
    from dioptrin_b200 import _native as N
    shape = (61, 67)
    plan = _plan(dg, shape)
    frames = _frames(shape, 4, np.uint16, seed=2)
    chunks = [dg.bslz4_compress(f) for f in frames]
    N.check(N.lib().dg_plan_profile(plan.handle, 1))
    plan.integrate_bslz4_stack(chunks, "uint16")
    ms, n = C.c_double(0), C.c_int64(0)
    N.check(N.lib().dg_plan_decode_time(plan.handle, 1, C.byref(ms), C.byref(n)))
    assert n.value == 1 and ms.value > 0
    gms, gl, launches = C.c_double(0), C.c_int64(0), C.c_int64(0)
    N.check(N.lib().dg_plan_kernel_time(plan.handle, 1, C.byref(gms), C.byref(gl),
                                        C.byref(launches)))
    assert launches.value == 3  # decode, gather, finalize
    plan.close()
