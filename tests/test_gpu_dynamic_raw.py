"""Per-frame masks (dg_integrate_dynamic; the reference's Dynamic1dPlan,
src/integration/dynamic.rs) and raw sums (dg_integrate_raw;
Integrator::integrate1d_raw*, src/integration/methods.rs:299-360) on the
device against the CPU oracle's raw row sums (row(), src/lut/prepared.rs:
1011-1118, strict FP64).

Intensity and sigma within 1e-5 relative (the FP32 weights and products of
the device, the magnitude-scaled test of the other parity tests); the
plan's own denominators and weight sums without per-frame masks are FP64 on
both sides."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5
SHAPE = (57, 71)
NB = 80
PONI = dict(pixel1=172e-6, pixel2=172e-6, distance=0.05, poni1=20.3 * 172e-6,
            poni2=30.7 * 172e-6, rot1=0.02, rot2=-0.015, wavelength=1e-10)


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


@pytest.fixture(scope="module")
def ref(oracle):
    p = oracle.poni(**PONI)
    table = oracle.build_ps1d(p, *SHAPE, NB)
    norm = oracle.centres(p, *SHAPE, polarization_factor=0.95)["norm"]
    return dict(table=table, norm=norm)


def _integrator(dg):
    return dg.Integrator.from_poni_dict(PONI, method="pixel_split", polarization_factor=0.95)


def _masks(n, seed, p=0.1):
    rng = np.random.default_rng(seed)
    m = (rng.random((n,) + SHAPE) < p).astype(np.uint8)
    m[:, 10, :] = 1          # a masked row in every frame
    m[0, :, :20] = 1         # a large masked region in frame 0
    return m


def _close(got, want, scale):
    fin = np.isfinite(want)
    assert np.array_equal(fin, np.isfinite(got)), "non-finite bins differ"
    np.testing.assert_allclose(got[fin], want[fin], rtol=TOL, atol=TOL * scale)


def _oracle_dynamic(oracle, ref, frame, mask):
    s, n, v, c = oracle.raw_sums(ref["table"], mask.ravel(), ref["norm"], frame.ravel())
    safe = np.where(n == 0, 1.0, n)
    i = np.where(n == 0, 0.0, s / safe)
    sg = np.sqrt(np.maximum(np.where(n == 0, 0.0, v / (safe * safe)), 0.0))
    return i, sg, (s, n, v, c)


# None: the plan's tuned mapping (entry-lane gather with per-frame masks);
# 8: the masked bin tiles on mapping 8's tiles.
VARIANTS = [None, 8]


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("dtype", ["uint16", "uint32", "int32", "float32", "float64"])
def test_dynamic_masks_match_the_oracle(dg, oracle, ref, dtype, variant):
    plan = _integrator(dg).prepare_dynamic1d(SHAPE, NB)
    if variant is not None:
        plan.cuda_plan.gather_variant = variant
    frames = np.random.default_rng(1).poisson(50.0, (5,) + SHAPE).astype(dtype)
    masks = _masks(5, 2)
    if dtype.startswith("float"):
        frames[1][masks[1] != 0] = np.nan   # masked NaN pixels add nothing
        frames[2, 30, 40] = np.nan          # an unmasked NaN reaches its bins
        masks[2, 30, 40] = 0
    I, S = plan.cuda_plan.integrate_dynamic_stack(frames, masks, errors=True)
    for k in range(5):
        i, sg, _ = _oracle_dynamic(oracle, ref, frames[k].astype(np.float64), masks[k])
        scale = np.nanmax(np.abs(i))
        _close(I[k], i, scale)
        _close(S[k], sg, np.nanmax(sg))
    plan.close()


@pytest.mark.parametrize("variant", VARIANTS)
def test_shared_mask_and_worker_api(dg, oracle, ref, variant):
    dyn = _integrator(dg).prepare_dynamic1d(SHAPE, NB)
    if variant is not None:
        dyn.cuda_plan.gather_variant = variant
    assert dyn.shape == SHAPE and dyn.n_points == NB
    frames = np.random.default_rng(3).poisson(30.0, (4,) + SHAPE).astype(np.uint32)
    mask = _masks(1, 4)[0]
    I1, S1 = dyn.cuda_plan.integrate_dynamic_stack(frames, mask, errors=True)
    I2, S2 = dyn.cuda_plan.integrate_dynamic_stack(frames, np.stack([mask] * 4), errors=True)
    assert np.array_equal(I1, I2) and np.array_equal(S1, S2)
    w = dyn.worker()
    r = w.integrate1d(frames[2], mask, errors=True)
    assert np.array_equal(r.intensity_array, I1[2]) and np.array_equal(r.errors_array, S1[2])
    assert np.array_equal(r.radial_array, dyn.cuda_plan.radial_array)
    # no mask: every pixel counts
    r0 = w.integrate1d(frames[0])
    i, _, _ = _oracle_dynamic(oracle, ref, frames[0].astype(np.float64), np.zeros(SHAPE, np.uint8))
    _close(r0.intensity_array, i, i.max())
    # everything masked: empty bins
    allm = w.integrate1d(frames[0], np.ones(SHAPE, np.uint8), errors=True)
    assert not allm.intensity_array.any() and not allm.errors_array.any()
    with pytest.raises(ValueError):
        w.integrate1d(frames[0], mask, azimuthal_std=True)
    with pytest.raises(ValueError):
        dyn.cuda_plan.integrate_dynamic_stack(frames, mask[:5])
    with pytest.raises(TypeError):
        dyn.cuda_plan.integrate_dynamic_stack(frames, mask.astype(np.int32))
    with pytest.raises(ValueError):
        dyn.worker(0)
    dyn.close()


def test_dynamic_with_the_plan_mask_equals_the_fixed_plan(dg):
    it = _integrator(dg)
    mask = _masks(1, 6)[0]
    it.set_mask(mask)
    fixed = it.prepare_cuda1d(SHAPE, NB)
    dyn = it.prepare_dynamic1d(SHAPE, NB)  # the stored mask is left out
    frames = np.random.default_rng(5).poisson(80.0, (3,) + SHAPE).astype(np.float32)
    fi, fs, _ = fixed.integrate_stack(frames, errors=True)
    di, ds = dyn.cuda_plan.integrate_dynamic_stack(frames, mask, errors=True)
    _close(di, fi, fi.max())
    _close(ds, fs, fs.max())
    fixed.close()
    dyn.close()


def test_dynamic_device_form_equals_host_form(dg):
    import ctypes as C
    import torch
    from dioptrin_b200 import _native as N
    dyn = _integrator(dg).prepare_dynamic1d(SHAPE, NB)
    frames = np.random.default_rng(7).poisson(20.0, (6,) + SHAPE).astype(np.int32)
    masks = _masks(6, 8)
    hi, hs = dyn.cuda_plan.integrate_dynamic_stack(frames, masks, errors=True)
    df, dm = torch.from_numpy(frames).cuda(), torch.from_numpy(masks).cuda()
    oi = torch.empty((6, NB), dtype=torch.float64, device="cuda")
    os_ = torch.empty_like(oi)
    stream = torch.cuda.current_stream().cuda_stream
    N.check(N.lib().dg_integrate_dynamic_device(
        dyn.cuda_plan.handle, C.c_void_p(df.data_ptr()), 2, 6, C.c_void_p(dm.data_ptr()),
        SHAPE[0] * SHAPE[1], N.DG_ERRORS, C.c_void_p(oi.data_ptr()), C.c_void_p(os_.data_ptr()),
        C.c_void_p(stream)))
    torch.cuda.synchronize()
    assert np.array_equal(oi.cpu().numpy(), hi) and np.array_equal(os_.cpu().numpy(), hs)
    dyn.close()


@pytest.mark.parametrize("variant", [None, 5, 7, 8])
@pytest.mark.parametrize("dtype", ["uint32", "float64"])
def test_raw_sums_with_the_plan_mask(dg, oracle, ref, dtype, variant):
    # None: the tuned mapping; 7 and 8: the bin tiles write the raw sums
    # themselves, from the accumulators their normalised results divide.
    it = _integrator(dg)
    mask = _masks(1, 9)[0]
    it.set_mask(mask)
    plan = it.prepare_cuda1d(SHAPE, NB)
    if variant is not None:
        plan.gather_variant = variant
    frames = np.random.default_rng(10).poisson(40.0, (3,) + SHAPE).astype(dtype)
    res = plan.integrate_raw_stack(frames, with_variance=True)
    _, _, _, den = plan.export_table(0)
    I, S, _ = plan.integrate_stack(frames, errors=True)
    for k, r in enumerate(res):
        s, n, v, c = oracle.raw_sums(ref["table"], mask.ravel(), ref["norm"],
                                     frames[k].astype(np.float64).ravel())
        _close(r.sum_signal, s, s.max())
        _close(r.sum_variance, v, v.max())
        assert np.array_equal(r.sum_norm, den)             # the plan's FP64 denominators
        np.testing.assert_allclose(r.sum_norm, n, rtol=1e-9, atol=1e-15)
        np.testing.assert_allclose(r.count, c, rtol=1e-9, atol=1e-15)
        i = np.where(r.sum_norm == 0, 0.0, r.sum_signal / np.where(r.sum_norm == 0, 1, r.sum_norm))
        _close(i, I[k], I[k].max())
        if variant in (7, 8):
            assert np.array_equal(i, I[k])
            safe = np.where(r.sum_norm == 0, 1, r.sum_norm)
            q = np.where(r.sum_norm == 0, 0.0, r.sum_variance / (safe * safe))
            assert np.array_equal(np.sqrt(np.maximum(q, 0.0)), S[k])
        assert np.array_equal(r.bins, plan.radial_array)
    # without variance
    r0 = plan.integrate1d_raw(frames[0])
    assert r0.sum_variance is None and np.array_equal(r0.sum_signal, res[0].sum_signal)
    plan.close()


@pytest.mark.parametrize("variant", VARIANTS)
def test_raw_sums_with_per_frame_masks(dg, oracle, ref, variant):
    plan = _integrator(dg).prepare_dynamic1d(SHAPE, NB).cuda_plan
    if variant is not None:
        plan.gather_variant = variant
    frames = np.random.default_rng(11).poisson(60.0, (4,) + SHAPE).astype(np.uint16)
    masks = _masks(4, 12)
    res = plan.integrate_raw_stack(frames, masks, with_variance=True)
    di, _ = plan.integrate_dynamic_stack(frames, masks)
    for k, r in enumerate(res):
        s, n, v, c = oracle.raw_sums(ref["table"], masks[k].ravel(), ref["norm"],
                                     frames[k].astype(np.float64).ravel())
        _close(r.sum_signal, s, s.max())
        _close(r.sum_norm, n, n.max())
        _close(r.sum_variance, v, v.max())
        _close(r.count, c, c.max())
        i = np.where(r.sum_norm == 0, 0.0, r.sum_signal / np.where(r.sum_norm == 0, 1, r.sum_norm))
        assert np.array_equal(i, di[k])  # the same device sums, divided the same way
    plan.close()


def test_integrator_raw_methods_and_2d(dg, oracle, ref):
    it = _integrator(dg)
    f = np.random.default_rng(13).poisson(25.0, SHAPE).astype(np.float64)
    r = it.integrate1d_raw(f, NB)
    rv = it.integrate1d_raw_with_variance(f, NB)
    s, n, v, c = oracle.raw_sums(ref["table"], None, ref["norm"], f.ravel())
    _close(r.sum_signal, s, s.max())
    _close(rv.sum_variance, v, v.max())
    assert r.sum_variance is None
    p2 = it.prepare_cuda2d(SHAPE, 20, 12)
    raw2 = p2.integrate_raw_stack(f, with_variance=True)[0]
    i2, s2, _ = p2.integrate_stack(f, errors=True)
    assert raw2.sum_signal.shape == (240,)
    i = np.where(raw2.sum_norm == 0, 0.0,
                 raw2.sum_signal / np.where(raw2.sum_norm == 0, 1, raw2.sum_norm))
    _close(i, i2[0], i2.max())
    p2.close()


@pytest.mark.parametrize("with_masks", [False, True])
def test_raw_sums_batch_equals_single_frames(dg, with_masks):
    # 40 frames: the raw finalize takes frames in groups of 32, so frames 33
    # and 39 sit in a later group than frame 0; each must equal its own call.
    plan = _integrator(dg).prepare_dynamic1d(SHAPE, NB).cuda_plan
    plan.gather_variant = 5
    frames = np.random.default_rng(21).poisson(45.0, (40,) + SHAPE).astype(np.uint32)
    masks = _masks(40, 22) if with_masks else None
    res = plan.integrate_raw_stack(frames, masks, with_variance=True)
    for k in (0, 33, 39):
        one = plan.integrate_raw_stack(frames[k:k + 1], None if masks is None else masks[k:k + 1],
                                       with_variance=True)[0]
        for a, b in ((res[k].sum_signal, one.sum_signal), (res[k].sum_norm, one.sum_norm),
                     (res[k].sum_variance, one.sum_variance), (res[k].count, one.count)):
            assert np.array_equal(a, b)
    plan.close()
