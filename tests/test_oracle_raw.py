"""The oracle's raw row sums (S, N, V, C) and per-frame-mask integration,
pinned to the reference's known answers for integrate1d_raw*
(src/lut/integrate.rs:682-797) and to its rule that a dynamic-mask plan
equals integration with that mask (src/integration/dynamic.rs:370-406)."""
import numpy as np
import pytest


def _lut(o, row_ptr, col, w=None):
    return o.Lut(np.array(row_ptr), np.array(col), None if w is None else np.array(w), 0.0, 1.0)


def test_raw_returns_sums(oracle):
    s, n, v, c = oracle.raw_sums(_lut(oracle, [0, 2], [0, 1]), None, [2.0, 4.0], [10.0, 20.0])
    assert (s[0], n[0], c[0]) == (30.0, 6.0, 2.0)
    assert s[0] / n[0] == 5.0


def test_raw_weighted(oracle):
    s, n, v, c = oracle.raw_sums(_lut(oracle, [0, 2], [0, 1], [0.5, 0.5]), None, [2.0, 4.0],
                                 [10.0, 20.0])
    assert (s[0], n[0], c[0]) == (15.0, 3.0, 1.0)


def test_raw_variance(oracle):
    _, _, v, _ = oracle.raw_sums(_lut(oracle, [0, 2], [0, 1], [0.25, 0.75]), None, [1.0, 1.0],
                                 [1.0, 3.0])
    assert abs(v[0] - (0.25 * 0.25 * 1.0 + 0.75 * 0.75 * 3.0)) < 1e-12


def test_raw_with_mask(oracle):
    s, n, _, c = oracle.raw_sums(_lut(oracle, [0, 3], [0, 1, 2]), np.array([0, 1, 0], np.uint8),
                                 [1.0, 1.0, 1.0], [10.0, 20.0, 30.0])
    assert (s[0], n[0], c[0]) == (40.0, 2.0, 2.0)


def test_raw_2d_rows_and_empty_bins(oracle):
    s, *_ = oracle.raw_sums(_lut(oracle, [0, 2, 4], [0, 1, 2, 3]), None, np.ones(4),
                            [10.0, 20.0, 30.0, 40.0])
    assert list(s) == [30.0, 70.0]
    s, n, _, c = oracle.raw_sums(_lut(oracle, [0, 0, 1], [0]), None, [1.0], [10.0])
    assert list(s) == [0.0, 10.0] and n[0] == 0.0 and c[0] == 0.0


@pytest.mark.parametrize("mask", [[0, 1], [1, 0], [0, 0], [1, 1]])
def test_dynamic_mask_equals_compacted_table(oracle, mask):
    # custom_dynamic_grid_validates_shapes_and_recovers_after_failed_frames:
    # every mask of a two-pixel frame against integration with that mask.
    lut = _lut(oracle, [0, 2, 4], [0, 1, 0, 1], [0.25, 0.5, 0.75, 0.5])
    norm = np.array([2.0, 4.0])
    sig = np.array([-4.0, 2.0])
    m = np.array(mask, np.uint8)
    s, n, v, _ = oracle.raw_sums(lut, m, norm, sig)
    table = oracle.compact(lut, m)
    y, e = oracle.integrate_strict(table, oracle.denominators(table, norm), sig, True)
    i = np.where(n == 0, 0.0, s / np.where(n == 0, 1.0, n))
    assert np.array_equal(i, y)
    sg = np.sqrt(np.maximum(np.where(n == 0, 0.0, v / np.where(n == 0, 1.0, n * n)), 0))
    assert np.allclose(sg, e, rtol=1e-15, atol=0)
