"""The oracle's 2D tables (integration/grid.rs, lut/shared_grid.rs,
lut/pyfai_split.rs, lut/supersampled.rs) against the reference's own 2D
known answers (integration/azimuthal_range_tests.rs)."""
import math

import numpy as np
import pytest

ROWS, COLS, NR, NA = 60, 80, 12, 18


def _poni(oracle):
    # azimuthal_range_tests.rs:13-26: beam inside the detector, slight tilt.
    return oracle.poni(pixel1=1e-4, pixel2=1e-4, distance=0.05, poni1=0.003, poni2=0.004,
                       rot1=0.01, rot2=-0.02, wavelength=1e-10)


def _row_sums(lut, signal):
    out = np.zeros(lut.n_rows)
    for r in range(lut.n_rows):
        a, b = lut.row_ptr[r], lut.row_ptr[r + 1]
        out[r] = np.sum(lut.w[a:b] * signal[lut.col[a:b]])
    return out


def test_grid_rejects_invalid_ranges(oracle):
    # azimuthal_range_tests.rs:514-527.
    for rng in [(math.nan, 1.0), (0.0, math.inf), (1.0, 1.0), (1.0, -1.0),
                (0.0, 2 * math.pi + 0.01), (-4 * math.pi, 4 * math.pi)]:
        with pytest.raises(ValueError):
            oracle.grid2d(NR, NA, (0.0, 1.0), rng)


def test_grid_corrects_distant_full_turns(oracle):
    # grid.rs:86-96, azimuthal_range_tests.rs:538-571: (-3pi, -pi) is (-pi, pi).
    g = oracle.grid2d(NR, NA, (0.0, 1.0), (-3 * math.pi, -math.pi))
    assert g.a0 == -math.pi and g.a1 == -math.pi + 2 * math.pi
    g = oracle.grid2d(NR, NA, (0.0, 1.0), (-7.0, -6.0))
    e = oracle.grid2d(NR, NA, (0.0, 1.0), (-7.0 + 2 * math.pi, -6.0 + 2 * math.pi))
    assert abs(g.a0 - e.a0) < 1e-15


def test_index_rounding_stays_in_the_last_bin(oracle):
    # azimuthal_range_tests.rs:391-448.
    n = NA
    found = None
    for k in range(1, 2000):
        lo = -math.pi + k * 1e-4
        hi = lo + 2.0
        step = (hi - lo) / n
        v = hi
        for _ in range(4):
            v = np.nextafter(v, -np.inf)
            if int((v - lo) / step) >= n:
                found = (lo, hi, v)
                break
        if found:
            break
    lo, hi, v = found
    plain = oracle.grid2d(NR, n, (0.0, 1.0), (lo, hi))
    assert plain.bin(0.5, v) is None
    plain.clamp_index_rounding = 1
    assert plain.bin(0.5, v) == (n - 1) * NR + NR // 2
    assert plain.bin(0.5, hi) is None
    assert plain.bin(0.5, lo - 1e-12) is None
    circle = oracle.grid2d(NR, n, (0.0, 1.0), (-math.pi, math.pi))
    circle.clamp_index_rounding = 1
    assert circle.bin(0.5, np.nextafter(-math.pi, -np.inf)) == (n - 1) * NR + NR // 2


def _unwrapped_azimuth(oracle, rng):
    # azimuthal_range_tests.rs:151-158: centre azimuths unwrapped around the
    # middle of the range.
    cc = oracle.centres(_poni(oracle), ROWS, COLS)["chi"]
    c = 0.5 * (rng[0] + rng[1])
    return c - math.pi + np.mod(cc - c + math.pi, 2 * math.pi)


def test_counting_puts_each_pixel_in_the_bin_holding_its_azimuth(oracle):
    # azimuthal_range_tests.rs:161-200.
    p = _poni(oracle)
    for rng in [(0.0, math.pi / 2), (2.5, 2.5 + math.pi / 2), (-math.pi, math.pi),
                (0.3, 0.3 + 2 * math.pi)]:
        g = oracle.grid2d_for(p, ROWS, COLS, "counting", NR, NA, unit="2th_deg",
                              azimuthal_range=rng)
        lut = oracle.build_2d(p, ROWS, COLS, "counting", g, unit="2th_deg")
        az = _unwrapped_azimuth(oracle, rng)
        norm = _row_sums(lut, np.ones(ROWS * COLS))
        sig = _row_sums(lut, az)
        step = (rng[1] - rng[0]) / NA
        full = rng[1] - rng[0] > 6.0
        filled = 0
        for ia in range(NA):
            lo = rng[0] + ia * step
            any_ = False
            for ir in range(NR):
                k = ia * NR + ir
                if norm[k] == 0 or (full and ia in (0, NA - 1)):
                    continue
                any_ = True
                mean = sig[k] / norm[k]
                assert lo - 1e-9 <= mean <= lo + step + 1e-9
            filled += any_
        assert filled >= NA - 2


@pytest.mark.parametrize("method", ["counting", "pixel_split", "supersampled", "pyfai_full"])
def test_sectors_exclude_pixels_outside_their_edges(oracle, method):
    # azimuthal_range_tests.rs:203-250 (pyfai_full added: its sector test is
    # the same vertex rule).
    p = _poni(oracle)
    tth = oracle.centres(p, ROWS, COLS)["radial"]
    radius_px = 0.05 * np.tan(tth) / 1e-4
    for rng in [(0.0, math.pi / 2), (2.5, 2.5 + math.pi / 2), (-2.0, -1.0)]:
        g = oracle.grid2d_for(p, ROWS, COLS, method, NR, NA, unit="2th_deg", n_ss=3,
                              azimuthal_range=rng)
        lut = oracle.build_2d(p, ROWS, COLS, method, g, unit="2th_deg", n_ss=3)
        az = _unwrapped_azimuth(oracle, rng)
        far = ((radius_px > 15.0) & ((az < rng[0] - 0.1) | (az > rng[1] + 0.1))).astype(float)
        assert far.sum() > 100
        assert np.all(_row_sums(lut, far) == 0.0)
        assert np.count_nonzero(_row_sums(lut, np.ones(ROWS * COLS)) > 0) > 40


@pytest.mark.parametrize("method", ["pixel_split", "supersampled", "pyfai_full"])
def test_full_circle_tables_conserve_every_pixel(oracle, method):
    # shared_grid.rs: fractional weights are area fractions of the pixel, the
    # supersampled ones count / n_ss^2, pyFAI's are normalised per pixel;
    # on a full circle and the default radial edges every pixel sums to one.
    p = _poni(oracle)
    g = oracle.grid2d_for(p, ROWS, COLS, method, NR, NA, unit="2th_deg", n_ss=3,
                          azimuthal_range=(-math.pi, math.pi))
    lut = oracle.build_2d(p, ROWS, COLS, method, g, unit="2th_deg", n_ss=3)
    totals = np.bincount(lut.col, weights=lut.w, minlength=ROWS * COLS)
    assert np.max(np.abs(totals - 1.0)) < 1e-9
    # rows list pixels in ascending order
    for r in range(lut.n_rows):
        c = lut.col[lut.row_ptr[r]:lut.row_ptr[r + 1]]
        assert np.all(np.diff(c) > 0)


def test_default_grids_follow_the_method_rules(oracle):
    # methods.rs:365-388, grid.rs:579-624: index rounding always; counting
    # clamps the radial end, supersampling both outside edges, pyfai_full
    # uses (-pi, pi) and the pyFAI histogram mode.
    p = _poni(oracle)
    g = oracle.grid2d_for(p, ROWS, COLS, "counting", NR, NA)
    assert (g.clamp_index_rounding, g.clamp_radial_end, g.clamp_radial_outside) == (1, 1, 0)
    g = oracle.grid2d_for(p, ROWS, COLS, "supersampled", NR, NA, n_ss=2)
    assert (g.clamp_radial_outside, g.clamp_azimuthal_outside) == (1, 1)
    g = oracle.grid2d_for(p, ROWS, COLS, "supersampled", NR, NA, n_ss=2,
                          azimuthal_range=(0.0, 1.0))
    assert (g.clamp_radial_outside, g.clamp_azimuthal_outside) == (1, 0)
    g = oracle.grid2d_for(p, ROWS, COLS, "pyfai_full", NR, NA)
    assert g.pyfai == 1 and g.a0 == -math.pi and g.a1 == math.pi
    g = oracle.grid2d_for(p, ROWS, COLS, "pixel_split", NR, NA, radial_range=(1.0, 20.0))
    assert (g.r0, g.r1, g.clamp_radial_end, g.clamp_radial_outside) == (1.0, 20.0, 0, 0)
