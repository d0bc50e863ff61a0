"""The allocation-free integration entry point against the regular one.

dg_integrate_device_noalloc is for callers that may not allocate device
memory while they integrate (a real-time acquisition loop with a fixed memory
budget, a thread that must not enter the CUDA allocator): it keeps its partial
sums in a fixed array inside the library instead of allocating them. Its
results must match dg_integrate_device's on the same plan and frames, within
the tolerance of the other parity tests, and keep matching on a second call in
a row (the array keeps the previous call's contents).

This file sorts last so a run that stops at the first failure has run every
other test before it; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative, as the intensity/sigma parity tests


def _poni():
    return dict(pixel1=172e-6, pixel2=172e-6, distance=0.08, poni1=60.3 * 172e-6,
                poni2=75.7 * 172e-6, rot1=0.02, rot2=-0.01, wavelength=1e-10)


def _run(fn, plan, frames, flags, nb):
    import torch
    n = frames.shape[0]
    oi = torch.full((n, nb), np.nan, dtype=torch.float64, device=frames.device)
    os_ = torch.full_like(oi, np.nan)
    od = torch.full_like(oi, np.nan)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    from dioptrin_b200 import _native as N
    N.check(fn(plan.handle, C.c_void_p(frames.data_ptr()), 1, n, flags,
               C.c_void_p(oi.data_ptr()), C.c_void_p(os_.data_ptr()), C.c_void_p(od.data_ptr()),
               C.c_void_p(stream.cuda_stream)))
    torch.cuda.synchronize()
    return oi.cpu().numpy(), os_.cpu().numpy(), od.cpu().numpy()


def _close(a, b):
    fin = np.isfinite(b)
    assert np.array_equal(fin, np.isfinite(a))
    np.testing.assert_allclose(a[fin], b[fin], rtol=TOL, atol=0)


def test_noalloc_entry_matches_the_regular_entry_twice_in_a_row():
    import torch
    import dioptrin_b200 as dg
    from dioptrin_b200 import _native as N
    if not dg.cuda_available():
        pytest.fail("CUDA device required: " + str(dg.cuda_info()))
    shape, nb = (160, 200), 300
    it = dg.Integrator.from_poni_dict(_poni(), method="pixel_split", polarization_factor=0.99)
    mask = np.zeros(shape, np.uint8)
    mask[40:43, :] = 1
    it.set_mask(mask)
    plan = it.prepare_cuda1d(shape, nb)
    L = N.lib()
    gen = np.random.default_rng(11)
    for flags in (N.DG_ERRORS | N.DG_AZIMUTHAL_STD, N.DG_ERRORS, 0):
        frames_a = torch.from_numpy(gen.poisson(300.0, (5,) + shape).astype(np.uint32)).cuda()
        frames_b = torch.from_numpy(gen.poisson(80.0, (3,) + shape).astype(np.uint32)).cuda()
        frames_c = torch.from_numpy(gen.poisson(50.0, (40,) + shape).astype(np.uint32)).cuda()
        for frames in (frames_a, frames_b, frames_c):  # calls in a row, different contents
            ref = _run(L.dg_integrate_device, plan, frames, flags, nb)
            got = _run(L.dg_integrate_device_noalloc, plan, frames, flags, nb)
            _close(got[0], ref[0])
            if flags & N.DG_ERRORS:
                _close(got[1], ref[1])
            if flags & N.DG_AZIMUTHAL_STD:
                _close(got[2], ref[2])
    plan.close()


def test_noalloc_entry_rejects_bad_arguments():
    import dioptrin_b200 as dg
    from dioptrin_b200 import _native as N
    if not dg.cuda_available():
        pytest.fail("CUDA device required: " + str(dg.cuda_info()))
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
