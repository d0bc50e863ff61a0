"""One plan used from several CUDA streams at once.

dg_integrate_device takes any stream, and the request loop's workers each
run on their own stream, so two integrations of one plan may be in flight on
different streams together. The entry-lane and frame-lane gathers keep
per-segment partial sums in one scratch array per plan; the plan orders
every use of it across streams (an event after each use, waited for by the
next use on another stream). Results must equal the same frames integrated
one call at a time, bit for bit."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE, NB = (120, 150), 90


@pytest.fixture(scope="module")
def dg():
    import dioptrin_b200 as d
    if not d.cuda_available():
        pytest.fail("CUDA device required for -m gpu tests: " + str(d.cuda_info()))
    return d


@pytest.mark.parametrize("variant", [2, 5, 8])
def test_one_plan_on_two_streams(dg, variant):
    import torch
    from dioptrin_b200 import _native as N
    poni = dict(pixel1=172e-6, pixel2=172e-6, distance=0.05, poni1=50.3 * 172e-6,
                poni2=70.7 * 172e-6, rot1=0.02, wavelength=1e-10)
    it = dg.Integrator.from_poni_dict(poni, method="pixel_split", polarization_factor=0.97)
    plan = it.prepare_cuda1d(SHAPE, NB)
    plan.gather_variant = variant
    rng = np.random.default_rng(variant)
    sets = [torch.from_numpy(rng.poisson(30.0 + 40 * k, (12,) + SHAPE).astype(np.uint32)).cuda()
            for k in range(2)]
    flags = N.DG_ERRORS | N.DG_AZIMUTHAL_STD
    L = N.lib()
    torch.cuda.synchronize()  # the frames' copies ran on torch's stream

    def run(frames, stream):
        out = [torch.empty((frames.shape[0], NB), dtype=torch.float64, device="cuda")
               for _ in range(3)]
        N.check(L.dg_integrate_device(plan.handle, C.c_void_p(frames.data_ptr()), N.DG_U32,
                                      frames.shape[0], flags,
                                      *[C.c_void_p(o.data_ptr()) for o in out],
                                      C.c_void_p(stream.cuda_stream)))
        return out

    # one call at a time on a stream of its own, read back after it finished
    lone = torch.cuda.Stream()
    want = []
    for f in sets:
        outs = run(f, lone)
        torch.cuda.synchronize()
        want.append([o.cpu().numpy() for o in outs])
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    torch.cuda.synchronize()
    got = []
    for rep in range(10):  # alternate the streams without host waits between
        got.append([(k, run(sets[k], streams[(rep + k) % 2])) for k in range(2)])
    torch.cuda.synchronize()
    for pairs in got:
        for k, outs in pairs:
            for o, w in zip(outs, want[k]):
                assert np.array_equal(o.cpu().numpy(), w, equal_nan=True)
    plan.close()
