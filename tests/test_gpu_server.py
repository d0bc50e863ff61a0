"""The request loop (continuous batching across plans) on the device.

Requests for several plans (1D and 2D, different shapes and bin counts)
arrive from two threads at once; the loop coalesces same-plan requests into
one launch and runs plans concurrently. Every result must equal the same
frame integrated alone through the loop, bit for bit (a frame's sums do not
depend on the frames launched with it), and match the oracle-checked
Integrator path of the same configuration."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


def _configs(dg):
    poni = dict(pixel1=1e-4, pixel2=1e-4, distance=0.05, poni1=0.003, poni2=0.004,
                rot1=0.01, wavelength=1e-10)
    a = dg.Integrator.from_poni_dict(poni, method="pixel_split", polarization_factor=0.99)
    b = dg.Integrator.from_poni_dict(poni, method="supersampled", n_ss=2)
    c = dg.Integrator.from_poni_dict(dict(poni, distance=0.07), method="counting")
    return [(1, a, (60, 80), 90, 0, np.uint32, True, True),
            (2, b, (60, 80), 24, 18, np.uint16, True, False),
            (3, c, (48, 64), 50, 0, np.float32, False, False)]


def test_mixed_stream_results_equal_the_frames_alone(dg):
    loop = dg.RequestLoop(max_inflight_frames=64, max_coalesce=16)
    cfgs = _configs(dg)
    for key, it, shape, nb, na, _, _, _ in cfgs:
        loop.register(key, it, shape, nb, n_azimuthal=na)
    rng = np.random.default_rng(12)
    work = []
    for i in range(60):
        key, it, shape, nb, na, dt, err, std = cfgs[i % 3]
        work.append((key, rng.poisson(100.0, shape).astype(dt), err, std))
    results = {}

    def producer(items):
        for idx, (key, frame, err, std) in items:
            t = loop.submit(key, frame, errors=err, azimuthal_std=std)
            results[idx] = (key, t, err, std)

    threads = [threading.Thread(target=producer, args=(list(enumerate(work))[k::2],))
               for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    mixed = {}
    for idx, (key, t, err, std) in results.items():
        mixed[idx] = loop.poll(t, key, errors=err, azimuthal_std=std)
    stats = loop.stats()
    assert stats["completed"] == 60 and stats["failed"] == 0
    # alone: one request in flight at a time
    for idx, (key, frame, err, std) in enumerate(work):
        t = loop.submit(key, frame, errors=err, azimuthal_std=std)
        alone = loop.poll(t, key, errors=err, azimuthal_std=std)
        for a, b in zip(mixed[idx][:3], alone[:3]):
            if a is None:
                assert b is None
            else:
                assert np.array_equal(a, b, equal_nan=True), (idx, key)
    # the Integrator path of the same configurations (the loop tunes its own
    # plans' lane mappings, which round differently within the tolerance)
    for idx in (0, 1, 2):
        key, it, shape, nb, na, dt, err, std = cfgs[idx]
        frame = work[idx][1]
        if na:
            r = it.integrate2d(frame, nb, na, err)
        else:
            r = it.integrate1d(frame, nb, err, azimuthal_std=std)
        want = r.intensity_array
        np.testing.assert_allclose(mixed[idx][0], want, rtol=1e-5,
                                   atol=1e-5 * np.abs(want).max())
    loop.close()


def test_borrowed_pinned_frames(dg):
    loop = dg.RequestLoop(max_inflight_frames=32, max_coalesce=8)
    key, it, shape, nb, na, dt, err, std = _configs(dg)[0]
    loop.register(key, it, shape, nb, n_azimuthal=na)
    rng = np.random.default_rng(3)
    frames = [rng.poisson(50.0, shape).astype(dt) for _ in range(12)]
    pinned = dg.alloc_pinned((12,) + shape, dt)
    pinned[:] = np.stack(frames)
    tickets = [loop.submit(key, pinned[k], errors=err, azimuthal_std=std, borrow=True)
               for k in range(12)]
    got = [loop.poll(t, key, errors=err, azimuthal_std=std) for t in tickets]
    for k in range(12):
        t = loop.submit(key, frames[k], errors=err, azimuthal_std=std)
        ref = loop.poll(t, key, errors=err, azimuthal_std=std)
        for a, b in zip(got[k][:3], ref[:3]):
            assert np.array_equal(a, b, equal_nan=True)
    assert not loop._borrowed
    with pytest.raises(ValueError):
        loop.submit(key, pinned[0][:, ::2], borrow=True)
    loop.close()


def test_reregistered_plan_is_rebuilt(dg):
    loop = dg.RequestLoop()
    poni = dict(pixel1=1e-4, pixel2=1e-4, distance=0.05, poni1=0.003, poni2=0.004,
                wavelength=1e-10)
    it = dg.Integrator.from_poni_dict(poni, method="pixel_split")
    loop.register(7, it, (40, 50), 30)
    frame = np.full((40, 50), 10.0, np.float32)
    a = loop.poll(loop.submit(7, frame), 7)[0]
    moved = dg.Integrator.from_poni_dict(dict(poni, distance=0.051), method="pixel_split")
    loop.register(7, moved, (40, 50), 30)
    b = loop.poll(loop.submit(7, frame), 7)[0]
    assert loop.stats()["plan_builds"] == 2
    ref = moved.integrate1d(frame, 30).intensity_array
    np.testing.assert_allclose(b, ref, rtol=1e-5)  # the loop's plan has its own mapping
    assert not np.array_equal(a, b)
    loop.close()


def test_plan_cache_evicts_by_memory_and_rebuilds_evicted_plans(dg):
    # Three plans of a few MB each under a byte budget that holds two: the
    # builder evicts the least recently used idle plan to admit a new one, an
    # evicted plan is rebuilt on its next request, and every result equals
    # the first one for the same frame.
    poni = dict(pixel1=1e-4, pixel2=1e-4, distance=0.05, poni1=0.0103, poni2=0.0124,
                rot1=0.01, wavelength=1e-10)
    shape = (200, 240)
    its = [dg.Integrator.from_poni_dict(dict(poni, distance=0.05 + 0.0005 * k),
                                        method="pixel_split") for k in range(3)]
    probe = dg.RequestLoop(max_coalesce=4)  # plan bytes include its partial sums
    probe.register(0, its[0], shape, 300)
    frame = np.random.default_rng(9).poisson(80.0, shape).astype(np.uint32)
    probe.poll(probe.submit(0, frame, errors=True), 0, errors=True)
    one = probe.stats()["cache_bytes"]
    probe.close()
    assert one > 0
    loop = dg.RequestLoop(cache_bytes=int(2.5 * one), max_coalesce=4)
    for k in range(3):
        loop.register(k, its[k], shape, 300)
    first = {}
    for rnd in range(3):
        for k in range(3):  # round robin over 3 plans: each request misses
            got = loop.poll(loop.submit(k, frame, errors=True), k, errors=True)
            if rnd == 0:
                first[k] = got
            else:
                for a, b in zip(got[:2], first[k][:2]):
                    assert np.array_equal(a, b)
    st = loop.stats()
    assert st["completed"] == 9 and st["failed"] == 0
    assert st["plan_builds"] == 9 and st["plan_evictions"] >= 7
    assert st["cache_bytes"] <= 2.5 * one
    for k in range(3):
        ref = its[k].integrate1d(frame, 300, True)
        np.testing.assert_allclose(first[k][0], ref.intensity_array, rtol=1e-5)
    loop.close()


def test_a_plan_that_fails_to_build_fails_its_requests_only(dg):
    loop = dg.RequestLoop()
    good = dg.Integrator.from_poni_dict(dict(pixel1=1e-4, pixel2=1e-4, distance=0.05,
                                             poni1=0.003, poni2=0.004, wavelength=1e-10),
                                        method="pixel_split")
    # q units need a wavelength; the Integrator checks it when the unit is
    # set, so the wavelength is cleared afterwards and the device build
    # rejects the configuration (check_configuration, cuda.rs:1001-1057)
    bad = dg.Integrator.from_poni_dict(dict(pixel1=1e-4, pixel2=1e-4, distance=0.05,
                                            poni1=0.003, poni2=0.004, wavelength=1e-10),
                                       method="pixel_split", unit="q_nm^-1")
    bad.poni.wavelength = 0.0
    loop.register(1, good, (40, 50), 30)
    loop.register(2, bad, (40, 50), 30)
    frame = np.ones((40, 50), np.float32)
    t_bad = loop.submit(2, frame)
    t_good = loop.submit(1, frame)
    assert np.isfinite(loop.poll(t_good, 1)[0]).all()
    with pytest.raises(ValueError, match="[Ww]avelength"):
        loop.poll(t_bad, 2)
    st = loop.stats()
    assert st["completed"] == 1 and st["failed"] == 1
    loop.close()
