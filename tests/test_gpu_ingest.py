"""Host-side ingestion around the gather: frames stored bottom row first
(InputOrder::FlipVertical, src/integration/fixed.rs:18-23; remapped columns,
src/integration/cuda/device.rs:506-528) and page-locked frame buffers
(alloc_pinned_batch, src/python/cuda.rs:808-870; is_pinned_host,
device.rs:1055-1078).

A FlipVertical plan remaps pixel indices only, so on row-flipped frames it
must reproduce the detector-order plan bit for bit, for every lane mapping,
Bitshuffle/LZ4 chunks, per-frame masks and raw sums."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (53, 61)
PONI = dict(pixel1=172e-6, pixel2=172e-6, distance=0.05, poni1=15.3 * 172e-6,
            poni2=40.7 * 172e-6, rot1=0.03, rot2=-0.01, rot3=0.02, wavelength=1e-10)


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


def _integrator(dg, mask=True):
    it = dg.Integrator.from_poni_dict(PONI, method="pixel_split", polarization_factor=0.97)
    if mask:
        m = np.zeros(SHAPE, np.uint8)
        m[3, :] = 1       # near the top: must follow the flip
        m[:, 17] = 1
        it.set_mask(m)
    return it


def _eq(a, b):
    for x, y in zip(a, b):
        assert (x is None) == (y is None)
        if x is not None:
            assert np.array_equal(x, y, equal_nan=True)


def _count(plan):
    import ctypes as C
    from dioptrin_b200 import _native as N
    cnt = C.c_int32(0)
    N.check(N.lib().dg_plan_variant(plan.handle, -1, None, C.byref(cnt)))
    return cnt.value


def test_flip_vertical_is_bit_exact_for_every_mapping(dg):
    it = _integrator(dg)
    det = it.prepare_cuda1d(SHAPE, 70)
    flip = it.prepare_cuda1d(SHAPE, 70, input_order="flip_vertical")
    assert np.array_equal(det.radial_array, flip.radial_array)
    frames = np.random.default_rng(1).poisson(40.0, (5,) + SHAPE).astype(np.float32)
    frames[2, 5, 9] = np.nan
    flipped = np.ascontiguousarray(frames[:, ::-1, :])
    for v in range(_count(det)):
        det.gather_variant = v
        flip.gather_variant = v
        for flags in [(False, False), (True, False), (True, True)]:
            _eq(flip.integrate_stack(flipped, *flags), det.integrate_stack(frames, *flags))
    det.close()
    flip.close()


def test_flip_vertical_bslz4_dynamic_raw_and_2d(dg):
    it = _integrator(dg)
    det = it.prepare_cuda1d(SHAPE, 70)
    flip = it.prepare_cuda1d(SHAPE, 70, input_order="flip_vertical")
    frames = np.random.default_rng(2).poisson(30.0, (4,) + SHAPE).astype(np.uint32)
    flipped = np.ascontiguousarray(frames[:, ::-1, :])
    # Bitshuffle/LZ4 chunks of the stored (flipped) frames
    _eq(flip.integrate_bslz4_stack([dg.bslz4_compress(f) for f in flipped], "uint32", True),
        det.integrate_bslz4_stack([dg.bslz4_compress(f) for f in frames], "uint32", True))
    # raw sums with the plan mask
    for a, b in zip(flip.integrate_raw_stack(flipped, with_variance=True),
                    det.integrate_raw_stack(frames, with_variance=True)):
        _eq((a.sum_signal, a.sum_norm, a.sum_variance, a.count),
            (b.sum_signal, b.sum_norm, b.sum_variance, b.count))
    # per-frame masks travel with the frames
    masks = (np.random.default_rng(3).random((4,) + SHAPE) < 0.1).astype(np.uint8)
    fm = np.ascontiguousarray(masks[:, ::-1, :])
    ddet = _integrator(dg, mask=False).prepare_dynamic1d(SHAPE, 70)
    dflip = _integrator(dg, mask=False).prepare_dynamic1d(SHAPE, 70, input_order="flip_vertical")
    _eq(dflip.cuda_plan.integrate_dynamic_stack(flipped, fm, True),
        ddet.cuda_plan.integrate_dynamic_stack(frames, masks, True))
    # 2D
    d2 = it.prepare_cuda2d(SHAPE, 24, 16)
    f2 = it.prepare_cuda2d(SHAPE, 24, 16, input_order="flip_vertical")
    _eq(f2.integrate_stack(flipped, True), d2.integrate_stack(frames, True))
    with pytest.raises(ValueError):
        it.prepare_cuda1d(SHAPE, 70, input_order="upside_down")
    for p in (det, flip, d2, f2):
        p.close()
    ddet.close()
    dflip.close()


@pytest.mark.parametrize("dtype", [None, "uint16", "int32", "float64"])
def test_pinned_batches(dg, dtype):
    plan = _integrator(dg).prepare_cuda1d(SHAPE, 70)
    buf = plan.alloc_pinned_batch(6, dtype)
    assert buf.shape == (6,) + SHAPE and buf.flags.writeable
    assert buf.dtype == np.dtype(dtype or "float32")
    assert dg.is_pinned(buf) and not dg.is_pinned(np.empty(10))
    src = np.random.default_rng(4).poisson(25.0, (6,) + SHAPE).astype(buf.dtype)
    buf[:] = src
    _eq(plan.integrate_stack(buf, True, True), plan.integrate_stack(src.copy(), True, True))
    res = plan.batch1d(buf, errors=True)
    assert np.array_equal(res[3].intensity_array, plan.integrate_stack(src, True)[0][3])
    with pytest.raises(TypeError):
        plan.alloc_pinned_batch(2, "int8")
    del buf
    plan.close()


def test_flip_vertical_per_frame_masks_on_bin_tiles(dg):
    # The masked bin tiles read each frame's mask at the pixel indices the
    # flip remapped; flipped frames with flipped masks must give the detector
    # order's results bit for bit, normalised and raw.
    det = _integrator(dg, mask=False).prepare_dynamic1d(SHAPE, 70)
    flip = _integrator(dg, mask=False).prepare_dynamic1d(SHAPE, 70, input_order="flip_vertical")
    for p in (det, flip):
        p.cuda_plan.gather_variant = 8
    frames = np.random.default_rng(6).poisson(35.0, (5,) + SHAPE).astype(np.uint32)
    masks = (np.random.default_rng(7).random((5,) + SHAPE) < 0.15).astype(np.uint8)
    ff = np.ascontiguousarray(frames[:, ::-1, :])
    fm = np.ascontiguousarray(masks[:, ::-1, :])
    _eq(flip.cuda_plan.integrate_dynamic_stack(ff, fm, True),
        det.cuda_plan.integrate_dynamic_stack(frames, masks, True))
    for a, b in zip(flip.cuda_plan.integrate_raw_stack(ff, fm, with_variance=True),
                    det.cuda_plan.integrate_raw_stack(frames, masks, with_variance=True)):
        _eq((a.sum_signal, a.sum_norm, a.sum_variance, a.count),
            (b.sum_signal, b.sum_norm, b.sum_variance, b.count))
    det.close()
    flip.close()


@pytest.mark.parametrize("dtype", [np.uint16, np.uint32, np.int32, np.float32, np.float64])
def test_host_frames_in_two_slot_chunks_equal_device_frames(dg, dtype):
    # dg_integrate copies host frames through two staging slots (the next
    # chunk crosses the host link while the current one is gathered). A
    # small chunk budget makes 11 frames take several chunks in both slots,
    # with a short last chunk; the results must equal the same frames
    # integrated from device memory in one call, bit for bit.
    import ctypes as C

    import torch
    from dioptrin_b200 import _native as N
    it = _integrator(dg)
    nb = 70
    per_frame = SHAPE[0] * SHAPE[1] * 8 + nb * 24
    plan = it.prepare_cuda1d(SHAPE, nb, max_batch_bytes=3 * per_frame)
    assert plan.max_batch_frames == 3
    gen = np.random.default_rng(5)
    frames = gen.poisson(60.0, (11,) + SHAPE).astype(dtype)
    flags = N.DG_ERRORS | N.DG_AZIMUTHAL_STD
    host = plan.integrate_stack(frames, errors=True, azimuthal_std=True)
    codes = {np.uint16: N.DG_U16, np.uint32: N.DG_U32, np.int32: N.DG_I32,
             np.float32: N.DG_F32, np.float64: N.DG_F64}
    tdt = {np.uint16: torch.uint16, np.uint32: torch.uint32, np.int32: torch.int32,
           np.float32: torch.float32, np.float64: torch.float64}[dtype]
    dev = torch.from_numpy(frames.view(np.int16) if dtype == np.uint16 else frames)
    dev = dev.view(tdt).cuda()
    out = [torch.full((11, nb), -7.0, dtype=torch.float64, device="cuda") for _ in range(3)]
    torch.cuda.synchronize()
    N.check(N.lib().dg_integrate_device(plan.handle, C.c_void_p(dev.data_ptr()), codes[dtype], 11,
                                        flags, *[C.c_void_p(o.data_ptr()) for o in out], None))
    torch.cuda.synchronize()
    _eq(host, [o.cpu().numpy() for o in out])
    # a second call reuses the slots and the copy stream
    _eq(plan.integrate_stack(frames, errors=True, azimuthal_std=True), host)
    plan.close()


@pytest.mark.parametrize("dtype", [np.uint32, np.float64])
def test_masked_and_raw_host_calls_in_two_slot_chunks(dg, dtype):
    # dg_integrate_dynamic and dg_integrate_raw stage host frames and their
    # per-frame masks through the same two slots; with a small chunk budget
    # 11 frames take several chunks. Results equal the device-memory calls
    # on the same frames and masks bit for bit, for per-frame masks, for one
    # shared mask and (raw sums) for none.
    import ctypes as C

    import torch
    from dioptrin_b200 import _native as N
    it = _integrator(dg, mask=False)
    nb = 70
    per_frame = SHAPE[0] * SHAPE[1] * 8 + nb * 24
    plan = it.prepare_cuda1d(SHAPE, nb, max_batch_bytes=4 * per_frame)
    gen = np.random.default_rng(9)
    n = 11
    frames = gen.poisson(50.0, (n,) + SHAPE).astype(dtype)
    masks = (gen.random((n,) + SHAPE) < 0.1).astype(np.uint8)
    code = N.DG_U32 if dtype == np.uint32 else N.DG_F64
    tdt = torch.uint32 if dtype == np.uint32 else torch.float64
    dframes = torch.from_numpy(frames).view(tdt).cuda()
    dmasks = torch.from_numpy(masks).cuda()
    npix = SHAPE[0] * SHAPE[1]
    L = N.lib()
    vp = C.c_void_p
    for mask_kind in ("per_frame", "shared", "none"):
        hm = masks if mask_kind == "per_frame" else masks[:1] if mask_kind == "shared" else None
        stride = npix if mask_kind == "per_frame" else 0
        dm = None if hm is None else vp(dmasks.data_ptr())
        hmp = None if hm is None else vp(np.ascontiguousarray(hm).ctypes.data)
        for raw in (False, True):
            if hm is None and not raw:
                continue  # per-frame-mask calls need a mask
            k = 4 if raw else 2
            host = [np.full((n, nb), -7.0) for _ in range(k)]
            dev = [torch.full((n, nb), -7.0, dtype=torch.float64, device="cuda") for _ in range(k)]
            hp = [h.ctypes.data_as(C.POINTER(C.c_double)) for h in host]
            dp = [vp(d.data_ptr()) for d in dev]
            torch.cuda.synchronize()
            if raw:
                N.check(L.dg_integrate_raw(plan.handle, vp(frames.ctypes.data), code, n, hmp, stride,
                                           N.DG_ERRORS, *hp))
                N.check(L.dg_integrate_raw_device(plan.handle, vp(dframes.data_ptr()), code, n, dm,
                                                  stride, N.DG_ERRORS, *dp, None))
            else:
                N.check(L.dg_integrate_dynamic(plan.handle, vp(frames.ctypes.data), code, n, hmp,
                                               stride, N.DG_ERRORS, *hp))
                N.check(L.dg_integrate_dynamic_device(plan.handle, vp(dframes.data_ptr()), code, n,
                                                      dm, stride, N.DG_ERRORS, *dp, None))
            torch.cuda.synchronize()
            _eq(host, [d.cpu().numpy() for d in dev])
    plan.close()
