"""2D tables and cakes on the device against the CPU oracle.

Row pointers and column indices bit-exact, weights within the tolerance of
the 1D tables (the device's corner angles are correctly rounded where the C
library may misround a last bit); cakes within the integration tolerance.
Geometry and ranges follow the reference's 2D tests
(integration/azimuthal_range_tests.rs)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_I = 1e-5
ROWS, COLS, NR, NA = 60, 80, 12, 18


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


def _poni_dict():
    return dict(pixel1=1e-4, pixel2=1e-4, distance=0.05, poni1=0.003, poni2=0.004,
                rot1=0.01, rot2=-0.02, wavelength=1e-10)


def _integrator(dg, method, rng=None, mask=None):
    it = dg.Integrator.from_poni_dict(_poni_dict(), method=method, polarization_factor=0.99,
                                      unit="2th_deg", radial_range=rng, n_ss=3)
    if mask is not None:
        it.set_mask(mask)
    return it


CASES = [(None, None), ((-math.pi, math.pi), None), ((0.0, math.pi / 2), None),
         ((2.5, 2.5 + math.pi / 2), None), (None, (1.0, 20.0)), ((-3 * math.pi, -math.pi), None)]


@pytest.mark.parametrize("method", ["counting", "pixel_split", "pyfai_full", "supersampled"])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_2d_tables_bit_exact(dg, oracle, method, case):
    az, rr = CASES[case]
    it = _integrator(dg, method, rr)
    plan = it.prepare_cuda2d((ROWS, COLS), NR, NA, azimuthal_range=az, keep_tables=True)
    p = oracle.poni(**_poni_dict())
    g = oracle.grid2d_for(p, ROWS, COLS, method, NR, NA, unit="2th_deg", n_ss=3,
                          radial_range=rr, azimuthal_range=az)
    ref = oracle.build_2d(p, ROWS, COLS, method, g, unit="2th_deg", n_ss=3)
    rp, col, w, _ = plan.export_table(1)
    assert np.array_equal(rp, ref.row_ptr), "row_ptr differs"
    assert np.array_equal(col, ref.col), "col differs"
    np.testing.assert_allclose(w, ref.w, rtol=1e-12, atol=2e-9)
    np.testing.assert_array_equal(np.array(plan.radial), g.radial_centres())
    np.testing.assert_array_equal(plan.azimuthal_array, g.azimuthal_centres())


@pytest.mark.parametrize("method", ["pixel_split", "pyfai_full", "supersampled"])
def test_2d_cake_matches_the_oracle(dg, oracle, method):
    mask = np.zeros((ROWS, COLS), np.uint8)
    mask[7, :] = 1
    it = _integrator(dg, method, mask=mask)
    az = (-math.pi, math.pi)
    plan = it.prepare_cuda2d((ROWS, COLS), NR, NA, azimuthal_range=az)
    p = oracle.poni(**_poni_dict())
    g = oracle.grid2d_for(p, ROWS, COLS, method, NR, NA, unit="2th_deg", n_ss=3,
                          azimuthal_range=az)
    ref = oracle.build_2d(p, ROWS, COLS, method, g, unit="2th_deg", n_ss=3)
    norm = oracle.centres(p, ROWS, COLS, unit="2th_deg", polarization_factor=0.99)["norm"]
    table = oracle.compact(ref, mask.ravel())
    den = oracle.denominators(table, norm)
    frames = np.random.default_rng(5).poisson(300.0, (3, ROWS, COLS)).astype(np.uint16)
    res = plan.batch2d(frames, errors=True)
    for k, r in enumerate(res):
        yi, ys = oracle.integrate_strict(table, den, frames[k].astype(np.float64).ravel(), True)
        np.testing.assert_allclose(r.intensity_array, yi, rtol=TOL_I, atol=1e-12)
        np.testing.assert_allclose(r.errors_array, ys, rtol=TOL_I, atol=1e-12)
        assert r.n_radial == NR and r.n_azimuthal == NA
    single = it.integrate2d(frames[1], NR, NA, True, az)
    np.testing.assert_array_equal(single.intensity_array, res[1].intensity_array)


def test_2d_rejects_bad_ranges_and_the_spread(dg):
    it = _integrator(dg, "pixel_split")
    with pytest.raises(ValueError):
        it.prepare_cuda2d((ROWS, COLS), NR, NA, azimuthal_range=(0.0, 2 * math.pi + 0.01))
    with pytest.raises(ValueError):
        it.prepare_cuda2d((ROWS, COLS), NR, NA, azimuthal_range=(1.0, 1.0))
    plan = it.prepare_cuda2d((ROWS, COLS), NR, NA)
    with pytest.raises(ValueError):  # the spread is defined for 1D tables only
        plan.integrate_stack(np.ones((1, ROWS, COLS), np.float32), azimuthal_std=True)
