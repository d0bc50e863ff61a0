"""Parity of the CUDA path (through the C ABI) against the CPU oracle.

Tables: row pointers and column indices must be bit-exact, f64 weights and
denominators within 1e-12 relative (the device's FP64 atan2/cos differ from
glibc in the last bits). Integration: the reference's magnitude-scaled test
(src/integration/cuda/tests.rs:206-227) with the tolerance of this build's
compensated FP32 path, 1e-5 relative to sum(w*|s|)/den for intensity and
sigma; the spread within 1e-5 relative of the FP64 oracle."""
import math

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


def small_poni():
    # 64 x 80 detector, beam inside it (singular pixel), tilted.
    return dict(pixel1=172e-6, pixel2=172e-6, distance=0.05, poni1=24.3 * 172e-6,
                poni2=36.7 * 172e-6, rot1=0.03, rot2=-0.02, rot3=0.01, wavelength=1e-10)


def oracle_table(o, poni, shape, method, n, unit="2th_rad", rng=None, n_ss=2):
    p = o.poni(**poni)
    if method == "pixel_split":
        return o.build_ps1d(p, *shape, n, unit=unit, radial_range=rng)
    if method == "counting":
        c = o.centres(p, *shape, unit=unit)
        return o.build_counting1d(c["radial"], n, rng)
    if method == "supersampled":
        return o.build_ss1d(p, *shape, n, n_ss, unit=unit, radial_range=rng)
    if method == "pyfai_full":
        return o.build_pf1d(p, *shape, n, unit=unit, radial_range=rng)
    raise ValueError(method)


def make_integrator(dg, poni, method, unit="2th_rad", rng=None, pol=0.99, n_ss=2, mask=None):
    it = dg.Integrator.from_poni_dict(poni, method=method, polarization_factor=pol, unit=unit,
                                      radial_range=rng, n_ss=n_ss)
    if mask is not None:
        it.set_mask(mask)
    return it


def check_tables(o, plan, ref, mask, norm):
    rp, col, w, _ = plan.export_table(1)
    assert np.array_equal(rp, ref.row_ptr), "unmasked row_ptr differs"
    assert np.array_equal(col, ref.col), "unmasked col_idx differs"
    ref_w = ref.w if ref.w is not None else np.ones(len(ref.col))
    # A weight is area/area_total from shoelace sums over absolute (r, chi)
    # coordinates, which amplify a last-bit corner difference up to ~1e7-fold.
    # glibc misrounds ~0.1% of the reference's corner atan2 values (the device
    # rounds correctly), so weights agree to ~1e-9 absolute, far below their
    # FP32 storage resolution; indices are compared exactly.
    np.testing.assert_allclose(w, ref_w, rtol=1e-12, atol=2e-9)
    refc = o.compact(ref, mask)
    rp, col, w, den = plan.export_table(0)
    assert np.array_equal(rp, refc.row_ptr), "masked row_ptr differs"
    assert np.array_equal(col, refc.col), "masked col_idx differs"
    ref_den = o.denominators(refc, norm)
    # sums of ~1e4 weights carrying the ~1e-9 absolute weight noise above
    np.testing.assert_allclose(den, ref_den, rtol=1e-10, atol=1e-300)
    return refc, ref_den


@pytest.mark.parametrize("method", ["pixel_split", "counting", "supersampled", "pyfai_full"])
@pytest.mark.parametrize("unit", ["2th_rad", "2th_deg", "q_nm^-1"])
@pytest.mark.parametrize("ranged", [False, True])
def test_table_bit_exact_small(dg, oracle, method, unit, ranged):
    poni = small_poni()
    shape = (64, 80)
    n = 120
    rng = None
    if ranged:
        c = oracle.centres(oracle.poni(**poni), *shape, unit=unit)["radial"]
        rng = (float(np.quantile(c, 0.05)), float(np.quantile(c, 0.8)))
    mask = np.zeros(shape, np.uint8)
    mask[10:13, :] = 1
    mask[:, 40] = 1
    it = make_integrator(dg, poni, method, unit, rng, mask=mask)
    plan = it.prepare_cuda1d(shape, n, keep_tables=True)
    ref = oracle_table(oracle, poni, shape, method, n, unit, rng)
    norm = oracle.centres(oracle.poni(**poni), *shape, unit=unit, polarization_factor=0.99)["norm"]
    check_tables(oracle, plan, ref, mask.ravel(), norm)
    radial = np.array(plan.radial)
    np.testing.assert_array_equal(radial, ref.bins())


def _scale(o, table, den, signal):
    s, _ = o.row_sums(table, np.abs(signal))
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(den != 0, s / np.where(den != 0, den, 1), 0.0)


@pytest.mark.parametrize("dtype", ["uint16", "uint32", "int32", "float32", "float64"])
def test_integration_matches_oracle(dg, oracle, dtype):
    poni = small_poni()
    shape = (64, 80)
    n = 100
    mask = np.zeros(shape, np.uint8)
    mask[5, :] = 1
    it = make_integrator(dg, poni, "pixel_split", mask=mask)
    plan = it.prepare_cuda1d(shape, n, keep_tables=True)
    ref = oracle_table(oracle, poni, shape, "pixel_split", n)
    p = oracle.poni(**poni)
    norm = oracle.centres(p, *shape, polarization_factor=0.99)["norm"]
    table = oracle.compact(ref, mask.ravel())
    den = oracle.denominators(table, norm)
    rng = np.random.default_rng(3)
    frames = rng.poisson(200.0, (3,) + shape).astype(dtype)
    if dtype in ("int32", "float32", "float64"):
        frames[0, 7, 7] = -5
    I, S, D = plan.integrate_stack(frames, errors=True, azimuthal_std=True)
    for k in range(len(frames)):
        sig = frames[k].astype(np.float64).ravel()
        yi, ys = oracle.integrate_strict(table, den, sig, True)
        scale = _scale(oracle, table, den, sig)
        assert np.all(np.abs(I[k] - yi) <= TOL_I * scale), f"frame {k} intensity"
        var = np.maximum(sig, 0)
        si, se, sd = oracle.azimuthal_std(ref, mask.ravel(), norm, sig, var)
        np.testing.assert_allclose(I[k], si, rtol=TOL_I, atol=0)
        np.testing.assert_allclose(S[k], se, rtol=TOL_I, atol=1e-12)
        fin = np.isfinite(sd)
        assert np.array_equal(fin, np.isfinite(D[k]))
        np.testing.assert_allclose(D[k][fin], sd[fin], rtol=TOL_STD, atol=1e-6 * np.nanmax(si))
    # errors-only path uses the strict denominators (normalize_bin)
    I2, S2, _ = plan.integrate_stack(frames, errors=True)
    for k in range(len(frames)):
        sig = frames[k].astype(np.float64).ravel()
        yi, ys = oracle.integrate_strict(table, den, sig, True)
        scale = _scale(oracle, table, den, sig)
        assert np.all(np.abs(I2[k] - yi) <= TOL_I * scale)
        np.testing.assert_allclose(S2[k], ys, rtol=TOL_I, atol=0)


@pytest.mark.parametrize("method", ["pyfai_full", "supersampled", "counting"])
def test_other_methods_integrate_like_the_oracle(dg, oracle, method):
    poni = small_poni()
    shape = (64, 80)
    n = 90
    mask = np.zeros(shape, np.uint8)
    mask[30, :] = 1
    it = make_integrator(dg, poni, method, mask=mask)
    plan = it.prepare_cuda1d(shape, n)
    ref = oracle_table(oracle, poni, shape, method, n)
    norm = oracle.centres(oracle.poni(**poni), *shape, polarization_factor=0.99)["norm"]
    table = oracle.compact(ref, mask.ravel())
    den = oracle.denominators(table, norm)
    frames = np.random.default_rng(17).poisson(120.0, (4,) + shape).astype(np.uint32)
    I, S, D = plan.integrate_stack(frames, errors=True, azimuthal_std=True)
    for k in range(len(frames)):
        sig = frames[k].astype(np.float64).ravel()
        yi, ys = oracle.integrate_strict(table, den, sig, True)
        scale = _scale(oracle, table, den, sig)
        assert np.all(np.abs(I[k] - yi) <= TOL_I * scale), f"{method} frame {k}"
        np.testing.assert_allclose(S[k], ys, rtol=TOL_I, atol=1e-12)
        si, se, sd = oracle.azimuthal_std(ref, mask.ravel(), norm, sig, sig)
        fin = np.isfinite(sd)
        assert np.array_equal(fin, np.isfinite(D[k]))
        np.testing.assert_allclose(D[k][fin], sd[fin], rtol=TOL_STD, atol=1e-6 * np.nanmax(si))


def test_batch_is_bit_identical_to_single_frames(dg):
    poni = small_poni()
    shape = (64, 80)
    it = make_integrator(dg, poni, "pixel_split")
    plan = it.prepare_cuda1d(shape, 90)
    frames = np.random.default_rng(5).poisson(50.0, (9,) + shape).astype(np.uint32)
    for flags in [(False, False), (True, False), (True, True)]:
        I, S, D = plan.integrate_stack(frames, *flags)
        for k in range(len(frames)):
            i1, s1, d1 = plan.integrate_stack(frames[k], *flags)
            assert np.array_equal(I[k], i1[0])
            if flags[0]:
                assert np.array_equal(S[k], s1[0])
            if flags[1]:
                assert np.array_equal(D[k], d1[0], equal_nan=True)


def test_empty_bins_follow_the_reference_rules(dg, oracle):
    # A radial range reaching beyond the detector leaves empty rows:
    # intensity 0, sigma 0, spread NaN (prepared.rs:985-996, azimuthal.rs:83-85).
    poni = small_poni()
    shape = (64, 80)
    c = oracle.centres(oracle.poni(**poni), *shape)["radial"]
    rng = (float(c.min()), float(c.max()) * 3)
    it = make_integrator(dg, poni, "pixel_split", rng=rng)
    plan = it.prepare_cuda1d(shape, 60)
    frame = np.full(shape, 10, np.uint32)
    I, S, D = plan.integrate_stack(frame, True, True)
    empty = np.diff(plan.export_table(0)[0]) == 0
    assert empty.any()
    assert np.all(I[0][empty] == 0) and np.all(S[0][empty] == 0)
    assert np.all(np.isnan(D[0][empty]))


def test_fully_masked_table_gives_zeros(dg):
    # src/integration/cuda/tests.rs:971.
    poni = small_poni()
    shape = (32, 40)
    it = make_integrator(dg, poni, "pixel_split", mask=np.ones(shape, np.uint8))
    plan = it.prepare_cuda1d(shape, 30)
    assert plan.table_entries == 0
    I, S, D = plan.integrate_stack(np.ones(shape, np.float32), True, True)
    assert np.all(I == 0) and np.all(S == 0) and np.all(np.isnan(D))


def test_nonfinite_pixels_are_skipped_by_the_spread(dg, oracle):
    poni = small_poni()
    shape = (32, 40)
    it = make_integrator(dg, poni, "pixel_split")
    plan = it.prepare_cuda1d(shape, 40, keep_tables=True)
    ref = oracle_table(oracle, poni, shape, "pixel_split", 40)
    norm = oracle.centres(oracle.poni(**poni), *shape, polarization_factor=0.99)["norm"]
    f = np.random.default_rng(9).uniform(10, 20, shape).astype(np.float32)
    f[3, 4] = np.nan
    f[20, 30] = np.inf
    I, _, D = plan.integrate_stack(f, False, True)
    si, _, sd = oracle.azimuthal_std(ref, None, norm, f.astype(np.float64).ravel())
    np.testing.assert_allclose(I[0], si, rtol=TOL_I)
    np.testing.assert_allclose(D[0], sd, rtol=TOL_STD, atol=1e-6)


def test_plan_rejects_bad_frames(dg):
    it = make_integrator(dg, small_poni(), "pixel_split")
    plan = it.prepare_cuda1d((32, 40), 30)
    with pytest.raises(ValueError):
        plan.integrate_stack(np.zeros((2, 32, 41), np.float32))
    with pytest.raises(TypeError):
        plan.integrate_stack(np.zeros((2, 32, 40), np.int8))
    # the plan survives a failed call (src/integration/cuda/tests.rs:849-895)
    I, _, _ = plan.integrate_stack(np.ones((1, 32, 40), np.float32))
    assert np.isfinite(I).all()


@pytest.mark.parametrize("name", ["pilatus1m_ps1250", "eiger4m_ps2000_b256"])
def test_full_size_tables_bit_exact(dg, oracle, name):
    from dioptrin_b200 import workloads as W
    w = W.WORKLOADS[name]
    it = dg.Integrator.from_poni_dict(w.poni_dict(), method=w.method,
                                      polarization_factor=w.polarization_factor)
    mask = w.mask()
    it.set_mask(mask)
    plan = it.prepare_cuda1d(w.shape, w.n_points, keep_tables=True)
    ref = oracle.build_ps1d(oracle.poni(**w.poni_dict()), w.dim1, w.dim2, w.n_points)
    norm = oracle.centres(oracle.poni(**w.poni_dict()), w.dim1, w.dim2,
                          polarization_factor=w.polarization_factor)["norm"]
    table, den = check_tables(oracle, plan, ref, mask.ravel(), norm)
    frames = W.frames_numpy(w, 2)
    I, S, D = plan.integrate_stack(frames, True, True)
    for k in range(2):
        sig = frames[k].astype(np.float64).ravel()
        yi, ys = oracle.integrate_strict(table, den, sig, True)
        nz = den != 0
        rel = np.abs(I[k][nz] - yi[nz]) / np.maximum(np.abs(yi[nz]), 1e-300)
        assert rel.max() <= TOL_I, rel.max()
        si, se, sd = oracle.azimuthal_std(ref, mask.ravel(), norm, sig, np.maximum(sig, 0))
        np.testing.assert_allclose(S[k], se, rtol=TOL_I, atol=0)
        fin = np.isfinite(sd)
        np.testing.assert_allclose(D[k][fin], sd[fin], rtol=TOL_STD, atol=0)
