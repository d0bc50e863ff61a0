"""The batch drivers and the row-flipped input order against the CPU oracle.

Integrator.batch1d and batch1d_iter (src/python/integrator.rs:1867, :2211)
integrate lists of arrays, possibly of several shapes, through device plans
cached per (shape, bins); results keep the input order and must equal the
oracle's integrate1d_with_errors / integrate1d_with_azimuthal_std of each
array. batch1d_iter also takes an iterator without a length and reports an
error raised by the source at that item's position, after the items before
it. A plan with InputOrder::FlipVertical (Cuda1dOptions::with_input_order,
src/integration/cuda.rs:174-182) integrates frames stored bottom row first:
on np.flipud of a frame it must give the oracle's result for the frame."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5

PONI = dict(pixel1=172e-6, pixel2=172e-6, distance=0.07, poni1=40.3 * 172e-6,
            poni2=55.7 * 172e-6, rot1=0.02, rot2=-0.015, rot3=0.01, wavelength=1e-10)


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


def _reference(o, shape, n, mask):
    p = o.poni(**PONI)
    full = o.build_ps1d(p, *shape, n)
    norm = o.centres(p, *shape, polarization_factor=0.98)["norm"]
    m = None if mask is None else mask.ravel()
    table = o.compact(full, m)
    return full, table, m, norm, o.denominators(table, norm)


def _check(o, ref, frame, res, errors, std):
    full, table, m, norm, den = ref
    sig = frame.astype(np.float64).ravel()
    if std:
        yi, ys, yd = o.azimuthal_std(full, m, norm, sig, np.maximum(sig, 0))
        fin = np.isfinite(yd)
        assert np.array_equal(fin, np.isfinite(res.azimuthal_std_array))
        np.testing.assert_allclose(res.azimuthal_std_array[fin], yd[fin], rtol=TOL, atol=0)
    else:
        yi, ys = o.integrate_strict(table, den, sig, True)
    np.testing.assert_allclose(res.intensity_array, yi, rtol=TOL, atol=0)
    if errors:
        np.testing.assert_allclose(res.errors_array, ys, rtol=TOL, atol=0)
    else:
        assert res.errors_array is None


def _integrator(dg, mask):
    it = dg.Integrator.from_poni_dict(PONI, method="pixel_split", polarization_factor=0.98)
    it.set_mask(mask)
    return it


@pytest.mark.parametrize("errors,std", [(True, False), (True, True), (False, False)])
def test_batch1d_arrays_of_two_shapes_match_the_oracle(dg, oracle, errors, std):
    shapes = [(96, 120), (80, 110)]
    masks = {s: np.zeros(s, np.uint8) for s in shapes}
    for s, m in masks.items():
        m[7, :] = 1
        m[:, 33] = 1
    n = 140
    gen = np.random.default_rng(21)
    # interleaved shapes: results must come back in input order
    frames = [gen.poisson(100.0 + 10 * k, shapes[k % 2]).astype(np.uint32) for k in range(7)]
    for shape in shapes:
        it = _integrator(dg, masks[shape])
        ref = _reference(oracle, shape, n, masks[shape])
        sel = [f for f in frames if f.shape == shape]
        out = it.batch1d(sel, n, errors, azimuthal_std=std)
        assert [r.filename for r in out] == [f"array_{k}" for k in range(len(sel))]
        for f, r in zip(sel, out):
            assert r.is_ok()
            _check(oracle, ref, f, r.result, errors, std)
    # one call over both shapes (plans cached per shape)
    mixed = dg.Integrator.from_poni_dict(PONI, method="pixel_split", polarization_factor=0.98)
    out = mixed.batch1d(frames, n, errors, azimuthal_std=std)
    assert len(out) == len(frames)
    for f, r in zip(frames, out):
        _check(oracle, _reference(oracle, f.shape, n, None), f, r.result, errors, std)


def test_batch1d_iter_streams_in_order_and_reports_source_errors(dg, oracle):
    shape, n = (96, 120), 130
    mask = np.zeros(shape, np.uint8)
    mask[50, :] = 1
    it = _integrator(dg, mask)
    ref = _reference(oracle, shape, n, mask)
    gen = np.random.default_rng(4)
    frames = [gen.poisson(60.0, shape).astype(np.int32) for _ in range(45)]

    # a list: progress is known; read_ahead (num_workers) of 8 gives 6 batches
    results = it.batch1d_iter(frames, n, True, num_workers=8)
    assert results.progress == 0.0
    got = list(results)
    assert results.progress == 1.0
    assert [r.filename for r in got] == [f"array_{k}" for k in range(45)]
    for f, r in zip(frames, got):
        _check(oracle, ref, f, r.result, True, False)

    # an iterator without a length whose 11th item fails
    def source():
        for k, f in enumerate(frames[:20]):
            if k == 10:
                raise RuntimeError("source failed at item 10")
            yield f

    results = it.batch1d_iter(source(), n, True, num_workers=4, azimuthal_std=True)
    assert results.progress is None
    seen = []
    with pytest.raises(RuntimeError, match="item 10"):
        for r in results:
            seen.append(r)
    assert len(seen) == 10
    for f, r in zip(frames, seen):
        _check(oracle, ref, f, r.result, True, True)


@pytest.mark.parametrize("variant", [2, 5, 8])
def test_flip_vertical_plan_on_flipped_frames_matches_the_oracle(dg, oracle, variant):
    shape, n = (120, 150), 110
    mask = np.zeros(shape, np.uint8)
    mask[4:6, :] = 1  # near the top edge of the detector
    mask[:, 90] = 1
    it = _integrator(dg, mask)
    plan = it.prepare_cuda1d(shape, n, input_order="flip_vertical")
    plan.gather_variant = variant
    ref = _reference(oracle, shape, n, mask)
    gen = np.random.default_rng(8 + variant)
    frames = gen.poisson(70.0, (70,) + shape).astype(np.uint32)
    stored = np.ascontiguousarray(frames[:, ::-1, :])  # bottom row first
    I, S, D = plan.integrate_stack(stored, errors=True, azimuthal_std=True)
    I2, S2, _ = plan.integrate_stack(stored, errors=True)

    class R:
        pass

    for k in (0, 31, 32, 63, 64, 69):
        res = R()
        res.intensity_array, res.errors_array, res.azimuthal_std_array = I[k], S[k], D[k]
        _check(oracle, ref, frames[k], res, True, True)
        res.intensity_array, res.errors_array = I2[k], S2[k]
        _check(oracle, ref, frames[k], res, True, False)
    plan.close()
