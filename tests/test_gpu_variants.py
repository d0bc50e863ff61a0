"""Every lane mapping of the gather against the CPU oracle, and the per-plan
autotuner.

The gather kernel has several lane mappings (entry slices per frame group,
frames per lane, entries in flight per lane) that a plan picks between by
timing them. They accumulate in different orders, so each must meet the
parity tolerance on its own, keep a frame's result independent of the batch
it travels in, and leave padded remainder lanes out of the sums (a NaN in
pixel 0 must only reach the bins that contain pixel 0)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_I = 1e-5
TOL_STD = 1e-5


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


def _poni():
    return dict(pixel1=172e-6, pixel2=172e-6, distance=0.06, poni1=70.3 * 172e-6,
                poni2=96.7 * 172e-6, rot1=0.03, rot2=-0.02, rot3=0.01, wavelength=1e-10)


def _variant_count(dg, plan):
    import ctypes as C
    from dioptrin_b200 import _native as N
    cur, cnt = C.c_int32(0), C.c_int32(0)
    N.check(N.lib().dg_plan_variant(plan.handle, -1, C.byref(cur), C.byref(cnt)))
    return cnt.value


@pytest.fixture(scope="module")
def case(dg, oracle):
    shape, n = (150, 190), 160
    poni = _poni()
    mask = np.zeros(shape, np.uint8)
    mask[37, :] = 1
    mask[:, 101:104] = 1
    it = dg.Integrator.from_poni_dict(poni, method="pixel_split", polarization_factor=0.99)
    it.set_mask(mask)
    plan = it.prepare_cuda1d(shape, n, keep_tables=True)
    p = oracle.poni(**poni)
    ref = oracle.build_ps1d(p, *shape, n)
    norm = oracle.centres(p, *shape, polarization_factor=0.99)["norm"]
    table = oracle.compact(ref, mask.ravel())
    den = oracle.denominators(table, norm)
    yield dict(plan=plan, ref=ref, norm=norm, table=table, den=den, mask=mask, shape=shape)
    plan.close()


def _check_frame(oracle, c, I, S, D, frame):
    sig = frame.astype(np.float64).ravel()
    yi, ys = oracle.integrate_strict(c["table"], c["den"], sig, True)
    fin = np.isfinite(yi)
    assert np.array_equal(fin, np.isfinite(I)), "non-finite bins differ"
    np.testing.assert_allclose(I[fin], yi[fin], rtol=TOL_I, atol=1e-12)
    np.testing.assert_allclose(S[fin], ys[fin], rtol=TOL_I, atol=1e-12)
    if D is not None:
        si, se, sd = oracle.azimuthal_std(c["ref"], c["mask"].ravel(), c["norm"], sig,
                                          np.maximum(sig, 0))
        f2 = np.isfinite(sd)
        assert np.array_equal(f2, np.isfinite(D))
        np.testing.assert_allclose(D[f2], sd[f2], rtol=TOL_STD, atol=1e-6 * np.nanmax(si))


@pytest.mark.parametrize("dtype", ["uint32", "float32"])
def test_every_mapping_matches_the_oracle(dg, oracle, case, dtype):
    plan = case["plan"]
    frames = np.random.default_rng(21).poisson(150.0, (6,) + case["shape"]).astype(dtype)
    for v in range(_variant_count(dg, plan)):
        plan.gather_variant = v
        assert plan.gather_variant == v
        for flags in [(True, False), (True, True)]:
            I, S, D = plan.integrate_stack(frames, *flags)
            for k in range(len(frames)):
                _check_frame(oracle, case, I[k], S[k], None if D is None else D[k], frames[k])
    plan.gather_variant = 0


def test_every_mapping_keeps_a_nan_in_its_own_bins(dg, oracle, case):
    # Remainder steps pad with pixel 0; a NaN there must not leak into the
    # bins that do not contain pixel 0 (integration.rs strict sums).
    plan = case["plan"]
    f = np.random.default_rng(4).uniform(5, 50, case["shape"]).astype(np.float32)
    f[0, 0] = np.nan
    for v in range(_variant_count(dg, plan)):
        plan.gather_variant = v
        I, S, _ = plan.integrate_stack(f, errors=True)
        _check_frame(oracle, case, I[0], S[0], None, f)
    plan.gather_variant = 0


def test_every_mapping_gives_batch_equal_to_single(dg, case):
    plan = case["plan"]
    # 70 frames: the finalize and the bin tiles take frames in groups of 32
    # and 64, so frames 35 and 69 sit in later groups than frame 0
    frames = np.random.default_rng(8).poisson(40.0, (70,) + case["shape"]).astype(np.uint16)
    for v in range(_variant_count(dg, plan)):
        plan.gather_variant = v
        for flags in [(False, False), (True, False), (True, True)]:
            I, S, D = plan.integrate_stack(frames, *flags)
            for k in (0, 35, 69):
                i1, s1, d1 = plan.integrate_stack(frames[k], *flags)
                assert np.array_equal(I[k], i1[0]), (v, flags, k)
                if flags[0]:
                    assert np.array_equal(S[k], s1[0])
                if flags[1]:
                    assert np.array_equal(D[k], d1[0], equal_nan=True)
    plan.gather_variant = 0


def test_autotune_keeps_a_valid_mapping(dg, oracle, case):
    import torch
    plan = case["plan"]
    frames = np.random.default_rng(2).poisson(100.0, (4,) + case["shape"]).astype(np.uint32)
    dev = torch.from_numpy(frames).cuda()
    v, ms = plan.autotune(dev, errors=True, azimuthal_std=True)
    assert 0 <= v < _variant_count(dg, plan) == len(ms)
    # every mapping runs on this table; the bin tiles (7, 8) are timed only
    # when a launch fills the GPU (4 frames fill less than half of a tile's
    # frames; -1: not timed)
    tiles = (7, 8)
    assert all(t > 0 for i, t in enumerate(ms) if i not in tiles)
    assert all(ms[i] == -1 for i in tiles)
    assert ms[v] == min(t for t in ms if t > 0)
    assert plan.gather_variant == v
    I, S, D = plan.integrate_stack(frames, True, True)
    for k in range(len(frames)):
        _check_frame(oracle, case, I[k], S[k], D[k], frames[k])
    with pytest.raises(ValueError):
        plan.gather_variant = 99
    plan.gather_variant = 0


@pytest.mark.parametrize("dtype", ["uint32", "float32"])
def test_every_mapping_is_exact_on_tiny_units(dg, oracle, dtype):
    # Many narrow bins on a small detector leave units of fewer entry pairs
    # than warps (empty pieces in the frame-lane gather) beside long ones;
    # every bin must still match the FP64 oracle to FP32 rounding.
    shape, n = (96, 120), 1500
    poni = dict(pixel1=172e-6, pixel2=172e-6, distance=0.03, poni1=50.2 * 172e-6,
                poni2=61.4 * 172e-6, rot1=0.04, wavelength=1e-10)
    it = dg.Integrator.from_poni_dict(poni, method="pixel_split")
    plan = it.prepare_cuda1d(shape, n)
    p = oracle.poni(**poni)
    table = oracle.build_ps1d(p, *shape, n)
    norm = oracle.centres(p, *shape)["norm"]
    den = oracle.denominators(table, norm)
    frames = (1e6 * (1 + 1e-3 * np.random.default_rng(6).standard_normal((3,) + shape)))
    frames = frames.astype(dtype)
    for v in range(_variant_count(dg, plan)):
        plan.gather_variant = v
        I, _, _ = plan.integrate_stack(frames, errors=True)
        for k in range(len(frames)):
            yi, _ = oracle.integrate_strict(table, den, frames[k].astype(np.float64).ravel(), True)
            ok = yi != 0
            assert np.array_equal(ok, I[k] != 0)
            rel = np.abs(I[k][ok] - yi[ok]) / np.abs(yi[ok])
            assert rel.max() < 1e-6, (v, k, float(rel.max()))
    plan.close()
