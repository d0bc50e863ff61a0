"""Several plans in one launch: the work-queue gather (dg_multi_integrate).

A persistent grid of row-warp CTAs claims (plan, row item) items from one
counter until every plan of the call is summed, each row's results written by
the CTA that sums it; the device work is a CUDA graph captured on the first
call and replayed after it. Each plan is summed as lane mapping 10 sums it, so
every item's results must equal dg_integrate_device on that plan with mapping
10 selected, bit for bit, whatever the other plans of the call and their
sizes, on the first (captured) call and on replays with other frames and frame
counts (one, two and several frames per pass); and they must match the CPU
oracle within the parity tolerance. A call whose items carry no frames does
nothing; bad calls are rejected and leave the plans usable."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PONI = dict(pixel1=172e-6, pixel2=172e-6, distance=0.06, poni1=40.3 * 172e-6,
            poni2=52.7 * 172e-6, rot1=0.02, rot2=-0.01, wavelength=1e-10)
PONI_B = dict(PONI, distance=0.09)


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


def _plans(dg):
    """Plans of very different sizes: 1D pixel split, 1D counting, 2D cake."""
    a = dg.Integrator.from_poni_dict(PONI, method="pixel_split", polarization_factor=0.98)
    m = np.zeros((150, 180), np.uint8)
    m[20, :] = 1
    a.set_mask(m)
    b = dg.Integrator.from_poni_dict(PONI_B, method="counting")
    c = dg.Integrator.from_poni_dict(PONI, method="supersampled", n_ss=2)
    return [(a.prepare_cuda1d((150, 180), 200, keep_tables=True), (150, 180), 200, a),
            (b.prepare_cuda1d((60, 70), 40, keep_tables=True), (60, 70), 40, b),
            (c.prepare_cuda2d((150, 180), 60, 36), (150, 180), 60 * 36, c)]


def _h(plan):
    h = plan.handle
    return h.value if isinstance(h, C.c_void_p) else h


def _multi():
    from dioptrin_b200 import _native as N
    h = C.c_void_p()
    N.check(N.lib().dg_multi_create(0, 8, C.byref(h)))
    return h


def _run_multi(h, items, dtype, flags):
    import torch
    from dioptrin_b200 import _native as N
    arr = (N.MultiItem * len(items))()
    outs = []
    for k, (plan, frames, nb) in enumerate(items):
        n = frames.shape[0]
        o = [torch.full((max(n, 1), nb), -7.0, dtype=torch.float64, device="cuda")
             for _ in range(3)]
        outs.append(o)
        arr[k] = N.MultiItem(_h(plan), frames.data_ptr(), n, o[0].data_ptr(),
                             o[1].data_ptr(), o[2].data_ptr())
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    N.check(N.lib().dg_multi_integrate(h, arr, len(items), dtype, flags,
                                       C.c_void_p(stream.cuda_stream)))
    torch.cuda.synchronize()
    return [[x.cpu().numpy() for x in o] for o in outs]


def _run_single(plan, frames, nb, dtype, flags):
    import torch
    from dioptrin_b200 import _native as N
    n = frames.shape[0]
    o = [torch.full((n, nb), -7.0, dtype=torch.float64, device="cuda") for _ in range(3)]
    torch.cuda.synchronize()
    N.check(N.lib().dg_integrate_device(plan.handle, C.c_void_p(frames.data_ptr()), dtype, n,
                                        flags, *[C.c_void_p(x.data_ptr()) for x in o], None))
    torch.cuda.synchronize()
    return [x.cpu().numpy() for x in o]


@pytest.mark.parametrize("flags", [1, 0])
def test_multi_equals_each_plan_alone(dg, flags):
    import torch
    from dioptrin_b200 import _native as N
    plans = _plans(dg)
    for p, _, _, _ in plans:
        p.gather_variant = 10
    h = _multi()
    gen = np.random.default_rng(5 + flags)
    for rnd, counts in enumerate([(5, 70, 3), (33, 1, 64), (0, 9, 2), (1, 2, 1)]):
        frames = [torch.from_numpy(gen.poisson(50.0 + 20 * k, (n,) + shape).astype(np.uint16))
                  .cuda() for k, ((_, shape, _, _), n) in enumerate(zip(plans, counts))]
        items = [(p, f, nb) for (p, _, nb, _), f in zip(plans, frames)]
        got = _run_multi(h, items, N.DG_U16, flags)
        for k, ((p, shape, nb, _), f) in enumerate(zip(plans, frames)):
            if f.shape[0] == 0:
                continue
            ref = _run_single(p, f, nb, N.DG_U16, flags)
            assert np.array_equal(got[k][0], ref[0]), (rnd, k)
            if flags & N.DG_ERRORS:
                assert np.array_equal(got[k][1], ref[1]), (rnd, k)
    N.lib().dg_multi_destroy(h)
    for p, _, _, _ in plans:
        p.close()


def test_resident_claiming_grid_equals_the_per_tile_grid(dg):
    # The claiming form (resident CTAs taking four tiles per atomic add) runs
    # only for batches beyond 2^24 tiles; the test hook forces it here.
    import torch
    from dioptrin_b200 import _native as N
    plans = _plans(dg)
    gen = np.random.default_rng(17)
    frames = [torch.from_numpy(gen.poisson(70.0, (n,) + shape).astype(np.uint16)).cuda()
              for (_, shape, _, _), n in zip(plans, (9, 3, 5))]
    items = [(p, f, nb) for (p, _, nb, _), f in zip(plans, frames)]
    h = _multi()
    direct = _run_multi(h, items, N.DG_U16, N.DG_ERRORS)
    N.check(N.lib().dg_multi_test_resident(h, 1))
    for _ in range(2):  # the captured graph replayed with the other grid
        resident = _run_multi(h, items, N.DG_U16, N.DG_ERRORS)
        for a, b in zip(direct, resident):
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    N.lib().dg_multi_destroy(h)
    for p, _, _, _ in plans:
        p.close()


def test_multi_with_the_spread_matches_the_oracle(dg, oracle):
    import torch
    from dioptrin_b200 import _native as N
    plans = _plans(dg)[:2]  # the spread is defined for 1D tables
    h = _multi()
    gen = np.random.default_rng(2)
    frames = [torch.from_numpy(gen.poisson(90.0, (n,) + shape).astype(np.float32)).cuda()
              for (_, shape, _, _), n in zip(plans, (40, 7))]
    flags = N.DG_ERRORS | N.DG_AZIMUTHAL_STD
    for _ in range(2):  # captured, then replayed
        got = _run_multi(h, [(p, f, nb) for (p, _, nb, _), f in zip(plans, frames)],
                         N.DG_F32, flags)
        for k, ((p, shape, nb, it), f) in enumerate(zip(plans, frames)):
            po = oracle.poni(**(PONI if k == 0 else PONI_B))
            full = (oracle.build_ps1d(po, *shape, nb) if k == 0
                    else oracle.build_counting1d(oracle.centres(po, *shape)["radial"], nb))
            mask = None if it._mask is None else it._mask.ravel()
            norm = oracle.centres(po, *shape,
                                  polarization_factor=0.98 if k == 0 else None)["norm"]
            host = f.cpu().numpy()
            for j in (0, f.shape[0] - 1):
                sig = host[j].astype(np.float64).ravel()
                yi, ys, yd = oracle.azimuthal_std(full, mask, norm, sig, np.maximum(sig, 0))
                np.testing.assert_allclose(got[k][0][j], yi, rtol=1e-5, atol=0)
                np.testing.assert_allclose(got[k][1][j], ys, rtol=1e-5, atol=0)
                fin = np.isfinite(yd)
                assert np.array_equal(fin, np.isfinite(got[k][2][j]))
                np.testing.assert_allclose(got[k][2][j][fin], yd[fin], rtol=1e-5, atol=0)
    N.lib().dg_multi_destroy(h)
    for p, _, _, _ in plans:
        p.close()


def test_multi_rejects_bad_calls_and_plans_stay_usable(dg):
    import torch
    from dioptrin_b200 import _native as N
    plans = _plans(dg)
    h = _multi()
    L = N.lib()
    p, shape, nb, _ = plans[0]
    f = torch.zeros((2,) + shape, dtype=torch.uint32, device="cuda")
    o = torch.zeros((2, nb), dtype=torch.float64, device="cuda")
    item = N.MultiItem(_h(p), f.data_ptr(), 2, o.data_ptr(), o.data_ptr(), o.data_ptr())
    two = (N.MultiItem * 2)(item, item)
    assert L.dg_multi_integrate(h, two, 2, N.DG_U32, 0, None) == N.DG_INVALID_INPUT
    assert "one item" in N.last_error()
    p2, shape2, nb2, _ = plans[2]
    f2 = torch.zeros((1,) + shape2, dtype=torch.uint32, device="cuda")
    o2 = torch.zeros((1, nb2), dtype=torch.float64, device="cuda")
    one = (N.MultiItem * 1)(N.MultiItem(_h(p2), f2.data_ptr(), 1, o2.data_ptr(),
                                        o2.data_ptr(), o2.data_ptr()))
    assert L.dg_multi_integrate(h, one, 1, N.DG_U32, N.DG_AZIMUTHAL_STD,
                                None) == N.DG_UNSUPPORTED
    big = (N.MultiItem * 1)(N.MultiItem(_h(p), f.data_ptr(), 257, o.data_ptr(), None, None))
    assert L.dg_multi_integrate(h, big, 1, N.DG_U32, 0, None) == N.DG_UNSUPPORTED
    nine = (N.MultiItem * 9)()
    assert L.dg_multi_integrate(h, nine, 9, N.DG_U32, 0, None) == N.DG_INVALID_INPUT
    assert L.dg_multi_integrate(h, None, 0, N.DG_U32, 0, None) == N.DG_OK
    # the plans still integrate, alone and through the multi
    torch.cuda.synchronize()
    ref = _run_single(p, f, nb, N.DG_U32, 0)
    assert np.all(ref[0] == 0)
    got = _run_multi(h, [(p, f, nb)], N.DG_U32, 0)
    assert np.all(got[0][0] == 0)
    N.lib().dg_multi_destroy(h)
    for q, _, _, _ in plans:
        q.close()
