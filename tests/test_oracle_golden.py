"""Pins the CPU oracle against the reference's own golden vectors and the
known answers of its unit tests. Each test names the reference test it
restates (file:line in the reference crate)."""
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "geometry_v1.npz")


def v1_poni(o):
    g = np.load(GOLDEN)
    return o.poni(**{k[5:]: float(g[k]) for k in g.files if k.startswith("poni_")}), g


def test_sample_positions_match_pyfai(oracle):
    # geometry.rs:789-805: x/y/z against pyFAI, tolerance 1e-10.
    p, g = v1_poni(oracle)
    x, y, z = oracle.sample_positions(p, 10, 20)
    assert np.max(np.abs(x - g["x_pyFAI"])) <= 1e-10
    assert np.max(np.abs(y - g["y_pyFAI"])) <= 1e-10
    assert np.max(np.abs(z - g["z_pyFAI"])) <= 1e-10


def test_tth_chi_solid_angle_polarization_match_pyfai(oracle):
    # geometry.rs:807-920: tth, azimuth, solid angle, polarization(0.99), 1e-6.
    p, g = v1_poni(oracle)
    c = oracle.centres(p, 10, 20, polarization_factor=0.99)
    assert np.max(np.abs(c["tth"] - g["tth_pyFAI"])) <= 1e-6
    assert np.max(np.abs(c["chi"] - g["azimuth_pyFAI"])) <= 1e-6
    assert np.max(np.abs(c["sa"] - g["solid_angle_pyFAI"])) <= 1e-6
    assert np.max(np.abs(c["pol"] - g["polarization_pyFAI"])) <= 1e-6
    np.testing.assert_array_equal(c["norm"], c["pol"] * c["sa"])


def test_tth_at_centres_matches_all(oracle):
    # geometry.rs:824-840: calc_tth on centres equals calc_tth_all.
    p, _ = v1_poni(oracle)
    i, j = np.meshgrid(np.arange(10), np.arange(20), indexing="ij")
    t, a = oracle.tth_chi_at(p, i.ravel() + 0.5, j.ravel() + 0.5)
    c = oracle.centres(p, 10, 20)
    np.testing.assert_array_equal(t, c["tth"])
    np.testing.assert_array_equal(a, c["chi"])


def _ramp(hi, n):
    return np.array([1.0 + (hi - 1.0) * i / (n - 1) for i in range(n)])


def test_counting_automatic_range_keeps_every_pixel(oracle):
    # counting_csr.rs:265-279.
    for hi in [3.0, 30.8, 60.0, 1234.5]:
        for n in [7, 100, 1000, 1500, 3000]:
            radial = np.array([1.0 + (hi - 1.0) * i / 4999.0 for i in range(5000)])
            lut = oracle.build_counting1d(radial, n)
            assert len(lut.col) == len(radial)
            assert 4999 in lut.col[lut.row_ptr[n - 1]:]


def test_counting_explicit_range_includes_both_limits(oracle):
    # counting_csr.rs:300-311.
    for hi in [3.0, 30.8, 60.0, 1234.5]:
        for n in [7, 100, 1000, 1500, 3000]:
            radial = np.array([1.0, hi, hi + hi * 1e-12, 1.0 - 1e-12])
            lut = oracle.build_counting1d(radial, n, (1.0, hi))
            assert list(lut.col) == [0, 1]
            assert lut.row_ptr[1] == 1 and lut.row_ptr[n - 1] == 1


def test_counting_explicit_range_drops_pixels_outside(oracle):
    # counting_csr.rs:313-319.
    radial = np.array([0.5, 1.5, 2.5, 3.5, 1.0, 3.0, -4.0, np.inf])
    lut = oracle.build_counting1d(radial, 2, (1.0, 3.0))
    assert list(lut.row_ptr) == [0, 2, 4]
    assert list(lut.col) == [1, 4, 2, 5]


def test_histogram_maximum_lands_in_last_bin(oracle):
    # histogram.rs:275-302 (through the counting table, the same bin rule).
    for hi in [3.0, 30.8, 60.0, 1234.5]:
        data = _ramp(hi, 4800)
        for n in [7, 100, 1000, 1500, 3000]:
            lut = oracle.build_counting1d(data, n)
            assert 4799 in lut.col[lut.row_ptr[n - 1]:lut.row_ptr[n]]


def _radial_strip(o, n, offset, distance):
    # pixel_split.rs:964-973.
    return o.poni(pixel1=1e-6, pixel2=1e-4, distance=distance, poni1=0.5e-6,
                  poni2=-offset * 1e-4, wavelength=1e-10), 1, n


def _extent(o, p, dim1, dim2, pixel):
    r, _ = o.corners(p, dim1, dim2)
    w = dim2 + 1
    b = pixel // dim2 * w + pixel % dim2
    vals = [r[b], r[b + 1], r[b + w + 1], r[b + w]]
    return min(vals), max(vals)


def _pixel_total(lut, pixel):
    return float(sum(w for c, w in zip(lut.col, lut.w) if c == pixel))


def test_ps_split_pixel_gets_fractions_of_its_own_area(oracle):
    # pixel_split.rs:1014-1031.
    for offset, dist in [(300.0, 1.0), (3000.0, 10.0)]:
        p, d1, d2 = _radial_strip(oracle, 1, offset, dist)
        lo, hi = _extent(oracle, p, d1, d2, 0)
        step = hi - lo
        lut = oracle.ps1d_fractions(p, d1, d2, 2, lo - 0.7 * step, step)
        assert lut.row_ptr[1] - lut.row_ptr[0] == 1 and lut.row_ptr[2] - lut.row_ptr[1] == 1
        w0, w1 = lut.w[0], lut.w[1]
        assert abs(w0 - 0.3) < 1e-3 and abs(w1 - 0.7) < 1e-3
        assert abs(w0 + w1 - 1.0) < 1e-12


def test_ps_fully_included_pixels_have_unit_total_weight(oracle):
    # pixel_split.rs:1033-1054.
    p = oracle.poni(pixel1=1.7e-4, pixel2=2.1e-4, distance=0.14, poni1=-0.003, poni2=-0.002,
                    rot1=0.007, rot2=-0.009, wavelength=1e-10)
    r, _ = oracle.corners(p, 23, 29)
    lo, hi = r.min(), r.max() + 10 * np.finfo(float).eps
    lut = oracle.ps1d_fractions(p, 23, 29, 40, lo, (hi - lo) / 40.0)
    totals = np.bincount(lut.col, weights=lut.w, minlength=23 * 29)
    assert np.max(np.abs(totals - 1.0)) < 1e-9


def test_ps_range_clipped_pixel_keeps_in_range_fraction(oracle):
    # pixel_split.rs:1056-1079.
    p, d1, d2 = _radial_strip(oracle, 1, 300.0, 1.0)
    lo, hi = _extent(oracle, p, d1, d2, 0)
    mx = lo + 0.4 * (hi - lo)
    mn = lo - (mx - lo)
    lut = oracle.ps1d_fractions(p, d1, d2, 4, mn, (mx - mn) / 4.0)
    assert abs(_pixel_total(lut, 0) - 0.4) < 1e-3
    lut = oracle.build_ps1d(p, d1, d2, 4, radial_range=(mn, mx))
    assert all(c == 0 for c in lut.col)
    assert lut.row_ptr[4] - lut.row_ptr[3] == 1
    assert abs(lut.w.sum() - 0.4) < 1e-3


def test_ps_bin_weights_follow_pixel_fractions(oracle):
    # pixel_split.rs:1081-1103.
    p, d1, d2 = _radial_strip(oracle, 5, 10.0, 0.1)
    lo1, hi1 = _extent(oracle, p, d1, d2, 1)
    lo3, hi3 = _extent(oracle, p, d1, d2, 3)
    mn, mx = 0.5 * (lo1 + hi1), 0.5 * (lo3 + hi3)
    lut = oracle.build_ps1d(p, d1, d2, 1, radial_range=(mn, mx))
    assert list(lut.col) == [1, 2, 3]
    assert abs(lut.w[1] - 1.0) < 1e-12
    total = lut.w.sum()
    for value, expected in zip(lut.w, [0.25, 0.5, 0.25]):
        assert abs(value / total - expected) < 0.01


def test_ps_beam_pixel_uses_detector_plane_fractions(oracle):
    # pixel_split.rs:1105-1135.
    p = oracle.poni(pixel1=1e-4, pixel2=1e-4, distance=0.1, poni1=4.3e-4, poni2=5.6e-4,
                    wavelength=1e-10)
    beam = 4 * 11 + 5
    r, _ = oracle.corners(p, 9, 11)
    hi = r.max() + 10 * np.finfo(float).eps
    n = 200
    step = hi / n
    lut = oracle.ps1d_fractions(p, 9, 11, n, 0.0, step)
    totals = np.bincount(lut.col, weights=lut.w, minlength=99)
    assert np.max(np.abs(totals - 1.0)) < 1e-9
    radius = 0.1 * math.tan(step)
    expected = math.pi * radius * radius / 1e-8
    assert lut.row_ptr[1] - lut.row_ptr[0] == 1
    assert lut.col[0] == beam
    assert abs(lut.w[0] / expected - 1.0) < 0.05


def _beam_geometry(o, poni1, poni2):
    # pixel_split.rs:1137-1147.
    return o.poni(pixel1=1e-4, pixel2=1e-4, distance=0.05, poni1=poni1, poni2=poni2,
                  wavelength=1e-10)


def test_ps_automatic_range_conserves_the_beam_pixel(oracle):
    # pixel_split.rs:1158-1176.
    beam = 4 * 11 + 5
    for poni1, poni2 in [(4.5e-4, 5.5e-4), (4.3e-4, 5.6e-4)]:
        p = _beam_geometry(oracle, poni1, poni2)
        lut = oracle.build_ps1d(p, 9, 11, 200, unit="2th_deg")
        assert abs(_pixel_total(lut, beam) - 1.0) < 1e-12
        totals = np.bincount(lut.col, weights=lut.w, minlength=99)
        assert np.max(np.abs(totals - 1.0)) < 1e-9


def test_ps_explicit_range_keeps_in_range_part_of_beam_pixel(oracle):
    # pixel_split.rs:1178-1192.
    p = _beam_geometry(oracle, 4.5e-4, 5.5e-4)
    beam = 4 * 11 + 5
    c = oracle.centres(p, 9, 11, unit="2th_deg")
    mn = math.degrees(math.atan(0.5e-4 / 0.05))
    mn = math.atan(0.5e-4 / 0.05) * (180.0 / math.pi)
    mx = c["radial"].max() * 2.0
    lut = oracle.build_ps1d(p, 9, 11, 200, unit="2th_deg", radial_range=(mn, mx))
    assert abs(_pixel_total(lut, beam) - (1.0 - math.pi / 4.0)) < 2e-3


def test_strict_sigma_weighted_and_unweighted(oracle):
    # lut/integrate.rs:583-611.
    lut = oracle.build_counting1d(np.array([0.1, 0.2]), 1)
    den = oracle.denominators(lut, np.ones(2))
    _, s = oracle.integrate_strict(lut, den, np.array([1.0, 3.0]))
    assert abs(s[0] - 1.0) < 1e-12
    lut = oracle.Lut(np.array([0, 2]), np.array([0, 1]), np.array([0.25, 0.75]), 0.0, 1.0)
    den = oracle.denominators(lut, np.ones(2))
    _, s = oracle.integrate_strict(lut, den, np.array([1.0, 3.0]))
    assert abs(s[0] - math.sqrt(0.25 * 0.25 * 1.0 + 0.75 * 0.75 * 3.0)) < 1e-12


def test_empty_bins_report_zero(oracle):
    # prepared.rs:985-996 normalize_bin: den == 0 gives intensity 0, sigma 0.
    lut = oracle.Lut(np.array([0, 0, 1]), np.array([0]), np.array([1.0]), 0.0, 1.0)
    den = oracle.denominators(lut, np.ones(1))
    y, s = oracle.integrate_strict(lut, den, np.array([5.0]))
    assert list(y) == [0.0, 5.0] and list(s) == [0.0, math.sqrt(5.0)]


def _one_bin(o, w=None):
    return o.Lut(np.array([0, 3]), np.array([0, 1, 2]), None if w is None else np.array(w),
                 0.0, 1.0)


def test_spread_corrected_weighted_population(oracle):
    # azimuthal.rs:134-151.
    lut = _one_bin(oracle, [0.5, 0.25, 1.0])
    y, e, s = oracle.azimuthal_std(lut, None, np.array([2.0, 4.0, 2.0]),
                                   np.array([4.0, 16.0, 16.0]), np.array([4.0, 16.0, 16.0]))
    assert list(y) == [5.5]
    assert abs(s[0] - math.sqrt(6.75)) < 1e-12
    assert abs(e[0] - math.sqrt(18.0) / 4.0) < 1e-12


def test_spread_stable_at_large_offset(oracle):
    # azimuthal.rs:153-168.
    lut = _one_bin(oracle)
    _, _, s = oracle.azimuthal_std(lut, None, np.ones(3), np.array([1e12 - 1, 1e12, 1e12 + 1]))
    assert abs(s[0] - math.sqrt(2.0 / 3.0)) < 1e-12
    _, e, s = oracle.azimuthal_std(lut, None, np.ones(3), np.array([6.0, 12.0, 24.0]))
    assert abs(s[0] - math.sqrt(56.0)) < 1e-12 and e is None


def test_spread_masks_invalid_pixels_and_empty_bins(oracle):
    # azimuthal.rs:170-199.
    lut = _one_bin(oracle)
    y, _, s = oracle.azimuthal_std(lut, np.array([0, 1, 0], np.uint8), np.full(3, 2.0),
                                   np.array([10.0, 1e6, np.nan]))
    assert list(y) == [5.0] and list(s) == [0.0]
    y, e, s = oracle.azimuthal_std(lut, np.ones(3, np.uint8), np.ones(3), np.full(3, 10.0),
                                   np.full(3, 10.0))
    assert list(y) == [0.0] and math.isnan(s[0]) and list(e) == [0.0]
    _, _, s = oracle.azimuthal_std(lut, None, np.array([0.0, -1.0, np.inf]), np.full(3, 10.0))
    assert math.isnan(s[0])


def test_spread_empty_rows_and_zero_fraction(oracle):
    # azimuthal.rs:201-214.
    lut = oracle.Lut(np.array([0, 0, 1]), np.array([0]), np.array([0.0]), 0.0, 1.0)
    y, _, s = oracle.azimuthal_std(lut, None, np.ones(1), np.array([42.0]))
    assert list(y) == [0.0, 0.0] and all(math.isnan(v) for v in s)


def test_spread_invariant_to_pixel_order(oracle):
    # azimuthal.rs:216-240.
    a = _one_bin(oracle, [0.1, 0.5, 1.0])
    b = oracle.Lut(np.array([0, 3]), np.array([2, 1, 0]), np.array([1.0, 0.5, 0.1]), 0.0, 1.0)
    sig, norm = np.array([-10.0, 60.0, 80.0]), np.array([1.0, 2.0, 4.0])
    sa = oracle.azimuthal_std(a, None, norm, sig)[2]
    sb = oracle.azimuthal_std(b, None, norm, sig)[2]
    assert abs(sa[0] - sb[0]) < 1e-12


def test_spread_constant_corrected_signal_is_zero(oracle):
    # azimuthal.rs:242-251.
    lut = _one_bin(oracle, [0.2, 0.7, 1.0])
    y, _, s = oracle.azimuthal_std(lut, None, np.array([1.0, 2.0, 4.0]),
                                   np.array([20.0, 40.0, 80.0]))
    assert list(y) == [20.0] and list(s) == [0.0]


def test_ss1d_counts_every_subpixel(oracle):
    # supersampled.rs exact path: full-range 1D weights are count / n_ss^2 and
    # each pixel's weights sum to one on the automatic range.
    p = oracle.poni(pixel1=1.0, pixel2=1.0, distance=1.0)
    lut = oracle.build_ss1d(p, 10, 10, 100, 2)
    totals = np.bincount(lut.col, weights=lut.w, minlength=100)
    assert np.max(np.abs(totals - 1.0)) < 1e-12
    assert set(np.round(lut.w * 4).astype(int)) <= {1, 2, 3, 4}


def test_pf_radial_line_weights_match_pyfai_golden(oracle):
    # pyfai_1d.rs:392-413: pyFAI fullSplit1D_engine weights of one pixel on
    # four bins over [0, 2].
    w = oracle.split1d([(0.1, 0.2), (1.2, 0.3), (1.8, 1.5), (0.4, 1.7)], 4, (0.0, 2.0))
    expected = [0.21462747684427036, 0.4066985688044358, 0.32228298342690204,
                0.05639097092439181]
    assert [b for b, _ in w] == [0, 1, 2, 3]
    assert all(abs(a - e) < 1e-7 for (_, a), e in zip(w, expected))


def test_pf_partial_radial_pixel_renormalizes_and_disjoint_sector_excludes(oracle):
    # pyfai_1d.rs:415-424.
    poly = [(-0.5, 0.1), (-0.5, 0.8), (0.75, 0.8), (0.75, 0.1)]
    w = oracle.split1d(poly, 4, (0.0, 2.0), (0.2, 0.4), sector=True)
    assert abs(sum(x for _, x in w) - 1.0) < 1e-12
    assert all(math.isfinite(x) and x > 0 for _, x in w)
    assert oracle.split1d(poly, 4, (0.0, 2.0), (1.0, 2.0), sector=True) == []


def test_pf_seam_test_uses_pyfai_operator_precedence(oracle):
    # pyfai_1d.rs:429-434: 0.5 * X - Y is negative for this folded quad.
    poly = [(1.0, -0.5), (1.2, -0.4), (2.0, 0.25), (2.2, 0.6)]
    assert oracle.split1d(poly, 10, (0.0, 3.0), (1.0, 2.0), sector=True) == []


def _beam_geometry(oracle, poni1, poni2):
    # pyfai_1d.rs:532-541: 9 x 11 detector, 100 um pixels, beam in pixel (4, 5).
    return oracle.poni(pixel1=1e-4, pixel2=1e-4, distance=0.05, poni1=poni1, poni2=poni2,
                       wavelength=1e-10)


def test_pf_automatic_range_conserves_the_beam_pixel(oracle):
    # pyfai_1d.rs:554-567.
    for poni1, poni2 in [(4.5e-4, 5.5e-4), (4.3e-4, 5.6e-4)]:
        lut = oracle.build_pf1d(_beam_geometry(oracle, poni1, poni2), 9, 11, 200, unit="2th_deg")
        totals = np.bincount(lut.col, weights=lut.w, minlength=99)
        assert abs(totals[4 * 11 + 5] - 1.0) < 1e-12
        assert np.max(np.abs(totals - 1.0)) < 1e-9


def test_pf_explicit_range_clips_the_beam_pixel(oracle):
    # pyfai_1d.rs:569-588 (radial part; the sector form is not on this path).
    p = _beam_geometry(oracle, 4.5e-4, 5.5e-4)
    auto = oracle.pyfai_radial_range(p, 9, 11, unit="2th_deg")
    lo = math.degrees(math.atan(0.5e-4 / 0.05))
    lut = oracle.build_pf1d(p, 9, 11, 200, unit="2th_deg", radial_range=(lo, auto[1]))
    total = np.bincount(lut.col, weights=lut.w, minlength=99)[4 * 11 + 5]
    assert abs(total - (1.0 - math.pi / 4.0)) < 2e-3
    lut = oracle.build_pf1d(p, 9, 11, 200, unit="2th_deg", radial_range=auto)
    assert np.bincount(lut.col, weights=lut.w, minlength=99)[4 * 11 + 5] == 0.0
