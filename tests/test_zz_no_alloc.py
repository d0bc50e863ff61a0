"""The allocation-free integration entry point against the regular one.

dg_integrate_device_noalloc is for callers that may not allocate device
memory while they integrate (a real-time acquisition loop with a fixed memory
budget, a thread that must not enter the CUDA allocator): it keeps its partial
sums in a fixed array inside the library instead of allocating them. It runs
the same kernels in the same order as dg_integrate_device, so its results must
equal dg_integrate_device's bit for bit (NaN where it has NaN), for every lane
mapping of the gather, and keep matching on a second call in a row (the array
keeps the previous call's contents). A plan whose partial sums need several
launches to fit the array, one whose single frame does not fit it, and a fresh
plan whose device memory must not grow are covered too.

This file sorts last so a run that stops at the first failure has run every
other test before it; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required: " + str(d.cuda_info()))
    return d


def _poni():
    return dict(pixel1=172e-6, pixel2=172e-6, distance=0.08, poni1=60.3 * 172e-6,
                poni2=75.7 * 172e-6, rot1=0.02, rot2=-0.01, wavelength=1e-10)


def _run(fn, plan, frames, flags, nb):
    import torch
    from dioptrin_b200 import _native as N
    codes = {torch.uint32: N.DG_U32, torch.float32: N.DG_F32}
    n = frames.shape[0]
    oi = torch.full((n, nb), -7.0, dtype=torch.float64, device=frames.device)
    os_ = torch.full_like(oi, -7.0)
    od = torch.full_like(oi, -7.0)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    N.check(fn(plan.handle, C.c_void_p(frames.data_ptr()), codes[frames.dtype], n, flags,
               C.c_void_p(oi.data_ptr()), C.c_void_p(os_.data_ptr()), C.c_void_p(od.data_ptr()),
               C.c_void_p(stream.cuda_stream)))
    torch.cuda.synchronize()
    return oi.cpu().numpy(), os_.cpu().numpy(), od.cpu().numpy()


def _same(got, ref, flags):
    from dioptrin_b200 import _native as N
    assert np.array_equal(got[0], ref[0], equal_nan=True)
    if flags & N.DG_ERRORS:
        assert np.array_equal(got[1], ref[1], equal_nan=True)
    if flags & N.DG_AZIMUTHAL_STD:
        assert np.array_equal(got[2], ref[2], equal_nan=True)


def test_noalloc_entry_matches_the_regular_entry_for_every_mapping(dg):
    import torch
    from dioptrin_b200 import _native as N
    shape, nb = (160, 200), 300
    it = dg.Integrator.from_poni_dict(_poni(), method="pixel_split", polarization_factor=0.99)
    mask = np.zeros(shape, np.uint8)
    mask[40:43, :] = 1
    it.set_mask(mask)
    L = N.lib()
    gen = np.random.default_rng(11)
    # A fresh plan: the allocation-free call runs first and must not grow the
    # plan's device memory (its partial sums live in the library's array).
    plan = it.prepare_cuda1d(shape, nb)
    warm = torch.from_numpy(gen.poisson(30.0, (2,) + shape).astype(np.uint32)).cuda()
    before = plan.info().device_bytes
    got = _run(L.dg_integrate_device_noalloc, plan, warm, N.DG_ERRORS | N.DG_AZIMUTHAL_STD, nb)
    assert plan.info().device_bytes == before
    ref = _run(L.dg_integrate_device, plan, warm, N.DG_ERRORS | N.DG_AZIMUTHAL_STD, nb)
    _same(got, ref, N.DG_ERRORS | N.DG_AZIMUTHAL_STD)
    count = C.c_int32(0)
    N.check(L.dg_plan_variant(plan.handle, -1, None, C.byref(count)))
    for v in range(count.value):
        plan.gather_variant = v
        for flags in (N.DG_ERRORS | N.DG_AZIMUTHAL_STD, N.DG_ERRORS, 0):
            frames_a = torch.from_numpy(gen.poisson(300.0, (5,) + shape).astype(np.uint32)).cuda()
            frames_b = torch.from_numpy(gen.poisson(80.0, (70,) + shape).astype(np.uint32)).cuda()
            for frames in (frames_a, frames_b):  # two calls in a row, different contents
                ref = _run(L.dg_integrate_device, plan, frames, flags, nb)
                got = _run(L.dg_integrate_device_noalloc, plan, frames, flags, nb)
                _same(got, ref, flags)
    plan.close()


def test_noalloc_entry_splits_launches_to_fit_its_array(dg):
    # Eiger-4M-shaped, 3000 bins, float frames with the spread: six partial
    # sums per segment and frame, a few MB per frame, so the 32 MiB array
    # holds only a few frames per launch and the call takes several launches.
    from dioptrin_b200 import _native as N
    from dioptrin_b200 import workloads as W
    w = W.EIGER_4M_F32
    it = dg.Integrator.from_poni_dict(w.poni_dict(), method=w.method,
                                      polarization_factor=w.polarization_factor)
    it.set_mask(w.mask())
    plan = it.prepare_cuda1d(w.shape, w.n_points)
    plan.gather_variant = 2
    frames = W.frames_torch(w, 24, kind=w.kind)
    flags = N.DG_ERRORS | N.DG_AZIMUTHAL_STD
    L = N.lib()
    for _ in range(2):
        ref = _run(L.dg_integrate_device, plan, frames, flags, w.n_points)
        got = _run(L.dg_integrate_device_noalloc, plan, frames, flags, w.n_points)
        _same(got, ref, flags)
    plan.close()


def test_noalloc_entry_rejects_a_plan_too_large_for_its_array(dg):
    import torch
    from dioptrin_b200 import _native as N
    # 60 000 thin radial bins counted on a 1500 x 1500 detector: each bin's
    # few dozen pixels lie in as many detector strips, so there are millions
    # of (bin, strip) segments, far beyond 32 MiB of partial sums for one
    # frame with the spread on float pixels (six sums per segment).
    poni = dict(pixel1=75e-6, pixel2=75e-6, distance=0.1, poni1=700.3 * 75e-6,
                poni2=760.7 * 75e-6, wavelength=1e-10)
    shape, nb = (1500, 1500), 60000
    it = dg.Integrator.from_poni_dict(poni, method="counting")
    plan = it.prepare_cuda1d(shape, nb)
    frames = torch.zeros((1,) + shape, dtype=torch.float32, device="cuda")
    L = N.lib()
    out = torch.empty((1, nb), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = L.dg_integrate_device_noalloc(plan.handle, C.c_void_p(frames.data_ptr()), N.DG_F32, 1,
                                       N.DG_ERRORS | N.DG_AZIMUTHAL_STD,
                                       *[C.c_void_p(out.data_ptr())] * 3, None)
    assert st == N.DG_UNSUPPORTED, N.last_error()
    assert "partial sums" in N.last_error()
    # the plan still integrates through the regular entry point
    ref = _run(L.dg_integrate_device, plan, frames, N.DG_ERRORS, nb)
    assert np.all(ref[0] == 0)
    plan.close()


def test_noalloc_entry_rejects_bad_arguments(dg):
    from dioptrin_b200 import _native as N
    L = N.lib()
    assert L.dg_integrate_device_noalloc(None, None, 1, 1, 0, None, None, None,
                                         None) == N.DG_INVALID_INPUT
    it = dg.Integrator.from_poni_dict(_poni(), method="pixel_split")
    plan = it.prepare_cuda1d((32, 40), 20)
    assert L.dg_integrate_device_noalloc(plan.handle, None, 9, 1, 0, None, None, None,
                                         None) == N.DG_INVALID_INPUT
    assert L.dg_integrate_device_noalloc(plan.handle, None, 1, 0, 0, None, None, None,
                                         None) == N.DG_OK
    plan.close()
