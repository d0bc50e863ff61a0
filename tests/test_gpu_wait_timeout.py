"""Failure detection of the bin-tile gathers (lane mappings 7 and 8).

Their warps hand chunks to one another through shared-memory barriers, and
every wait gives up after 1 s, marking a flag in mapped host memory that the
host reads. dg_plan_test_wait_timeout runs one gather in which one warp of
one CTA never reports a chunk summed, so the other warps' waits run out: the
call must return DG_TIMEOUT after about a second, and the device context, the
plan and every later call must still work and give the same results as
before. No GPU fault is involved: the waits end by themselves."""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE, NB = (300, 320), 40


def _plan(dg):
    poni = dict(pixel1=172e-6, pixel2=172e-6, distance=0.05, poni1=120.3 * 172e-6,
                poni2=140.7 * 172e-6, rot1=0.02, rot2=-0.01, wavelength=1e-10)
    it = dg.Integrator.from_poni_dict(poni, method="pixel_split", polarization_factor=0.98)
    return it.prepare_cuda1d(SHAPE, NB)


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


def _ptr(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("variant", [7, 8])
def test_expired_wait_is_reported_and_the_plan_recovers(dg, variant):
    import torch
    from dioptrin_b200 import _native as N
    L = N.lib()
    plan = _plan(dg)
    plan.gather_variant = variant
    frames_np = np.random.default_rng(variant).poisson(50.0, (8,) + SHAPE).astype(np.uint32)
    want = plan.integrate_stack(frames_np, True, True)
    frames = torch.from_numpy(frames_np).cuda()
    out = [torch.full((8, NB), np.nan, dtype=torch.float64, device="cuda") for _ in range(3)]
    flags = N.DG_ERRORS | N.DG_AZIMUTHAL_STD
    torch.cuda.synchronize()
    t0 = time.monotonic()
    st = L.dg_plan_test_wait_timeout(plan.handle, _ptr(frames), N.DG_U32, 8, flags,
                                     *[_ptr(o) for o in out])
    took = time.monotonic() - t0
    assert st == N.DG_TIMEOUT, (st, N.last_error())
    assert "gave up" in N.last_error()
    assert 0.9 < took < 30.0
    # the context and the plan work on, with the results of before
    got = plan.integrate_stack(frames_np, True, True)
    for a, b in zip(got, want):
        assert np.array_equal(a, b, equal_nan=True)
    N.check(L.dg_integrate_device(plan.handle, _ptr(frames), N.DG_U32, 8, flags,
                                  *[_ptr(o) for o in out], None))
    torch.cuda.synchronize()
    for o, b in zip(out, want):
        assert np.array_equal(o.cpu().numpy(), b, equal_nan=True)
    plan.close()


def test_mappings_without_a_chunk_pipeline_are_rejected(dg):
    import torch
    from dioptrin_b200 import _native as N
    plan = _plan(dg)
    plan.gather_variant = 2
    frames = torch.zeros((2,) + SHAPE, dtype=torch.int32, device="cuda")
    out = torch.zeros((2, NB), dtype=torch.float64, device="cuda")
    st = N.lib().dg_plan_test_wait_timeout(plan.handle, _ptr(frames), N.DG_I32, 2, 0, _ptr(out),
                                           None, None)
    assert st == N.DG_UNSUPPORTED
    assert "mapping 7 or 8" in N.last_error()
    plan.close()
