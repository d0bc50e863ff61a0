"""Full-size parity of the benchmarked configurations: the lane mappings the
benchmark runs, on the benchmark's detectors, tables and batch sizes, checked
frame by frame against the CPU oracle.

1D batches (the bin tiles of lane mapping 8: 16-bin tiles x 64 frames, every
chunk ring and frame group exercised):
  - Pilatus-1M-shaped, 1250 bins, 256 int32 frames, errors;
  - Eiger-4M-shaped, 2000 bins, 256 uint32 frames, errors + azimuthal spread;
  - the precision stress case: Eiger-4M geometry, 3000 bins, 128 float32
    frames of 1e6 background, errors + azimuthal spread.
Every frame is compared with the oracle's strict FP64 sums (normalize_bin,
prepared.rs:985-1118) or, with the spread, its two-pass FP64 spread
(azimuthal.rs:48-118), relative error <= 1e-5 for intensity, sigma and the
spread, with the empty-bin rules (I = 0, sigma = 0, spread NaN).

2D cakes (Eiger-9M-shaped, 1000 x 360 bins over chi -pi..pi with the seam
across the detector, supersampled n_ss=4 and pyfai_full): row pointers and
column indices of the device tables bit-exact against the oracle's builders
(shared_grid.rs:13-232, pyfai_split.rs:35-168, supersampled.rs:1437-1477),
and the entry-lane gather of lane mapping 2 against the oracle on uint16
frames.

Few-frame launches: the row warps (mapping 10, the plain path's launch) on
the Eiger-4M table with the spread and on the 2D cake, and the entry-lane
mapping 3 that the cake's 64-frame batches pick."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_I = 1e-5     # intensity and sigma, relative to the FP64 oracle
TOL_STD = 1e-5   # azimuthal spread, relative to the FP64 oracle


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


def _oracle_setup(o, w):
    p = o.poni(**w.poni_dict())
    if w.n_azimuthal:
        g = o.grid2d_for(p, w.dim1, w.dim2, w.method, w.n_points, w.n_azimuthal,
                         n_ss=w.n_ss or 1, azimuthal_range=w.azimuthal_range)
        full = o.build_2d(p, w.dim1, w.dim2, w.method, g, n_ss=w.n_ss or 1)
    else:
        full = o.build_ps1d(p, w.dim1, w.dim2, w.n_points)
    mask = w.mask().ravel()
    norm = o.centres(p, w.dim1, w.dim2, polarization_factor=w.polarization_factor)["norm"]
    table = o.compact(full, mask)
    return full, table, mask, norm, o.denominators(table, norm)


def _plan(dg, w, keep_tables=False):
    it = dg.Integrator.from_poni_dict(w.poni_dict(), method=w.method, n_ss=w.n_ss,
                                      polarization_factor=w.polarization_factor)
    it.set_mask(w.mask())
    if w.n_azimuthal:
        return it.prepare_cuda2d(w.shape, w.n_points, w.n_azimuthal,
                                 azimuthal_range=w.azimuthal_range, keep_tables=keep_tables)
    return it.prepare_cuda1d(w.shape, w.n_points, keep_tables=keep_tables)


def _integrate_device(plan, frames, flags, nb):
    """dg_integrate_device on device-resident frames; results to the host."""
    import ctypes as C

    import torch
    from dioptrin_b200 import _native as N
    codes = {torch.uint16: N.DG_U16, torch.uint32: N.DG_U32, torch.int32: N.DG_I32,
             torch.float32: N.DG_F32, torch.float64: N.DG_F64}
    n = frames.shape[0]
    out = [torch.full((n, nb), -7.0, dtype=torch.float64, device=frames.device)
           for _ in range(3)]
    torch.cuda.synchronize()
    N.check(N.lib().dg_integrate_device(plan.handle, C.c_void_p(frames.data_ptr()),
                                        codes[frames.dtype], n, flags,
                                        *[C.c_void_p(o.data_ptr()) for o in out], None))
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in out]


def _rel(got, ref, sel):
    return np.abs(got[sel] - ref[sel]) / np.abs(ref[sel])


@pytest.mark.parametrize("name", ["pilatus1m_ps1250", "eiger4m_ps2000_b256",
                                  "eiger4m_ps3000_f32"])
def test_bin_tiles_full_size_every_frame(dg, oracle, name):
    from dioptrin_b200 import _native as N
    from dioptrin_b200 import workloads as W
    w = W.WORKLOADS[name]
    full, table, mask, norm, den = _oracle_setup(oracle, w)
    plan = _plan(dg, w)
    plan.gather_variant = 8
    assert plan.gather_variant == 8
    frames = W.frames_torch(w, w.n_frames, kind=w.kind)
    flags = (N.DG_ERRORS if w.errors else 0) | (N.DG_AZIMUTHAL_STD if w.azimuthal_std else 0)
    gi, gs, gd = _integrate_device(plan, frames, flags, plan.n_points)
    host = frames.cpu().numpy()
    del frames
    yi, ys, yd = oracle.integrate_frames_mt(table, den, full, mask, norm, host, w.errors,
                                            w.azimuthal_std, os.cpu_count() or 1)
    report = {}
    if w.azimuthal_std:
        # intensity and sigma of the spread path (sum c*s / sum w over valid entries)
        valid = np.isfinite(yd)
        assert np.array_equal(valid, np.isfinite(gd)), "NaN pattern of the spread differs"
        nz = yi != 0
        report["intensity"] = _rel(gi, yi, nz).max()
        report["sigma"] = _rel(gs, ys, ys != 0).max()
        report["azimuthal_std"] = _rel(gd, yd, valid & (yd != 0)).max()
        # empty bins: I = 0, sigma = 0, spread NaN (azimuthal.rs:83-85)
        assert np.all(gi[~valid] == 0) and np.all(gs[~valid] == 0)
        assert np.all(yi[~nz] == gi[~nz])
    else:
        nz = np.broadcast_to(den != 0, gi.shape)
        report["intensity"] = _rel(gi, yi, nz).max()
        report["sigma"] = _rel(gs, ys, nz & (ys != 0)).max()
        # empty bins: I = 0, sigma = 0 (prepared.rs:985-996)
        assert np.all(gi[~nz] == 0) and np.all(gs[~nz] == 0)
    print(name, {k: f"{v:.3g}" for k, v in report.items()})
    assert report["intensity"] <= TOL_I, report
    assert report["sigma"] <= TOL_I, report
    if w.azimuthal_std:
        assert report["azimuthal_std"] <= TOL_STD, report
    plan.close()


@pytest.mark.parametrize("name", ["eiger9m_2d_ss4", "eiger9m_2d_pyfai"])
def test_2d_cake_full_size(dg, oracle, name):
    from dioptrin_b200 import _native as N
    from dioptrin_b200 import workloads as W
    w = W.WORKLOADS[name]
    full, table, mask, norm, den = _oracle_setup(oracle, w)
    plan = _plan(dg, w, keep_tables=True)
    rp, col, wt, _ = plan.export_table(1)
    assert np.array_equal(rp, full.row_ptr), "unmasked row_ptr differs"
    assert np.array_equal(col, full.col), "unmasked col_idx differs"
    np.testing.assert_allclose(wt, full.w, rtol=1e-12, atol=2e-9)
    rp, col, _, dden = plan.export_table(0)
    assert np.array_equal(rp, table.row_ptr), "masked row_ptr differs"
    assert np.array_equal(col, table.col), "masked col_idx differs"
    np.testing.assert_allclose(dden, den, rtol=1e-10, atol=1e-300)
    plan.gather_variant = 2
    n = 16
    frames = W.frames_torch(w, n, kind=w.kind)
    nb = w.n_points * w.n_azimuthal
    gi, gs, _ = _integrate_device(plan, frames, N.DG_ERRORS, nb)
    host = frames.cpu().numpy()
    yi, ys, _ = oracle.integrate_frames_mt(table, den, full, mask, norm, host, True, False,
                                           os.cpu_count() or 1)
    nz = np.broadcast_to(den != 0, gi.shape)
    ri, rs = _rel(gi, yi, nz & (yi != 0)).max(), _rel(gs, ys, nz & (ys != 0)).max()
    print(name, f"intensity {ri:.3g} sigma {rs:.3g}")
    assert ri <= TOL_I and rs <= TOL_I
    assert np.all(gi[~nz] == 0) and np.all(gs[~nz] == 0)
    plan.close()


@pytest.mark.parametrize("name,n,variant", [("eiger4m_ps2000_b256", 3, 10),
                                            ("eiger9m_2d_ss4", 5, 10),
                                            ("eiger9m_2d_ss4", 9, 3)])
def test_few_frame_launches_full_size(dg, oracle, name, n, variant):
    """The few-frame launches on the benchmark's tables: the row warps
    (mapping 10: rows of more than 512 entries one per CTA on Eiger-4M,
    rows of at most 64 entries eight lanes each on the 2D cake, a pass of
    four frames and a partial second pass) and the entry-lane mapping the
    2D cake's batches pick, against the oracle frame by frame."""
    from dioptrin_b200 import _native as N
    from dioptrin_b200 import workloads as W
    w = W.WORKLOADS[name]
    full, table, mask, norm, den = _oracle_setup(oracle, w)
    plan = _plan(dg, w)
    plan.gather_variant = variant
    assert plan.gather_variant == variant
    frames = W.frames_torch(w, n, kind=w.kind)
    flags = (N.DG_ERRORS if w.errors else 0) | (N.DG_AZIMUTHAL_STD if w.azimuthal_std else 0)
    nb = w.n_points * max(1, w.n_azimuthal)
    gi, gs, gd = _integrate_device(plan, frames, flags, nb)
    host = frames.cpu().numpy()
    yi, ys, yd = oracle.integrate_frames_mt(table, den, full, mask, norm, host, w.errors,
                                            w.azimuthal_std, os.cpu_count() or 1)
    if w.azimuthal_std:
        valid = np.isfinite(yd)
        assert np.array_equal(valid, np.isfinite(gd)), "NaN pattern of the spread differs"
        assert _rel(gd, yd, valid & (yd != 0)).max() <= TOL_STD
        assert np.all(gi[~valid] == 0) and np.all(gs[~valid] == 0)
        nz = yi != 0
    else:
        nz = np.broadcast_to(den != 0, gi.shape)
        assert np.all(gi[~nz] == 0) and np.all(gs[~nz] == 0)
    assert _rel(gi, yi, nz & (yi != 0)).max() <= TOL_I
    assert _rel(gs, ys, nz & (ys != 0)).max() <= TOL_I
    plan.close()
