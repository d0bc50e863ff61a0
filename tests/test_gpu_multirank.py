"""Plan replicas on two ranks: each rank (one process, gloo for the host-side
exchange) builds its own plan of the same geometry on its GPU, integrates its
contiguous shard of the batch through dg_integrate_device, and rank 0 gathers
the shards. The gathered results must equal one process integrating the whole
batch with its own plan, bit for bit, for the bin tiles (lane mapping 8) and
the entry-lane units (lane mapping 0), and match the CPU oracle. Frames never
interact (src/batch.rs:69-101), so no collective sits on the data path; the
only device collective is the max over ranks of the device-timed elapsed time.

With one GPU both ranks share it. Their kernels never wait on one another:
each launch completes on its own, and the ranks meet only on the host."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE, N_BINS, N_FRAMES = (200, 240), 180, 37


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _poni():
    return dict(pixel1=172e-6, pixel2=172e-6, distance=0.07, poni1=80.3 * 172e-6,
                poni2=95.6 * 172e-6, rot1=0.015, rot2=-0.01, wavelength=1e-10)


def _frames():
    return np.random.default_rng(23).poisson(40.0, (N_FRAMES,) + SHAPE).astype(np.uint32)


def _integrate(plan, frames_np, device):
    import ctypes as C

    import torch
    from dioptrin_b200 import _native as N
    frames = torch.from_numpy(frames_np).to(device)
    n = frames.shape[0]
    out = [torch.full((n, N_BINS), -7.0, dtype=torch.float64, device=device) for _ in range(3)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    start.record()
    N.check(N.lib().dg_integrate_device(
        plan.handle, C.c_void_p(frames.data_ptr()), N.DG_U32, n,
        N.DG_ERRORS | N.DG_AZIMUTHAL_STD, *[C.c_void_p(o.data_ptr()) for o in out],
        C.c_void_p(torch.cuda.current_stream(device).cuda_stream)))
    stop.record()
    torch.cuda.synchronize(device)
    return [o.cpu().numpy() for o in out], start.elapsed_time(stop)


def _rank_main(rank, world, port, variant, out):
    import datetime

    import torch
    import torch.distributed as dist
    import dioptrin_b200 as dg
    from dioptrin_b200.sharding import max_over_ranks, shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        device = torch.device("cuda", rank % torch.cuda.device_count())
        torch.cuda.set_device(device)
        it = dg.Integrator.from_poni_dict(_poni(), method="pixel_split",
                                          polarization_factor=0.99)
        plan = it.prepare_cuda1d(SHAPE, N_BINS, device=device.index)
        plan.gather_variant = variant
        frames = _frames()
        a, b = shard(len(frames), rank, world)
        mine, ms = _integrate(plan, frames[a:b], device)
        gathered = [None] * world
        dist.all_gather_object(gathered, (a, b, mine))
        slowest = max_over_ranks(ms)
        if rank == 0:
            whole, _ = _integrate(plan, frames, device)
            parts = sorted(gathered, key=lambda g: g[0])
            got = [np.concatenate([p[2][k] for p in parts]) for k in range(3)]
            same = all(np.array_equal(x, y, equal_nan=True) for x, y in zip(got, whole))
            out.put((same, [p[:2] for p in parts], slowest >= ms, got))
        plan.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("variant", [8, 0])
def test_plan_replicas_on_two_ranks_match_one_process(oracle, variant):
    import dioptrin_b200 as dg
    if not dg.cuda_available():
        pytest.fail("CUDA device required: " + str(dg.cuda_info()))
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, variant, out)) for r in range(2)]
    for p in procs:
        p.start()
    result = out.get(timeout=300)
    for p in procs:
        p.join(60)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    same, spans, slowest_ok, (gi, gs, gd) = result
    assert spans == [(0, 19), (19, 37)]
    assert same, "sharded results differ from one process"
    assert slowest_ok
    # and against the oracle's FP64 sums and two-pass spread
    o = oracle
    p = o.poni(**_poni())
    full = o.build_ps1d(p, SHAPE[0], SHAPE[1], N_BINS)
    mask = np.zeros(SHAPE[0] * SHAPE[1], np.uint8)
    norm = o.centres(p, SHAPE[0], SHAPE[1], polarization_factor=0.99)["norm"]
    table = o.compact(full, mask)
    den = o.denominators(table, norm)
    yi, ys, yd = o.integrate_frames_mt(table, den, full, mask, norm,
                                       _frames().reshape(N_FRAMES, -1), True, True,
                                       os.cpu_count() or 1)
    nz = yi != 0
    assert np.all(np.abs(gi[nz] - yi[nz]) <= 1e-5 * np.abs(yi[nz]))
    assert np.all(gi[~nz] == 0)
    valid = np.isfinite(yd)
    assert np.array_equal(valid, np.isfinite(gd))
    sel = valid & (yd != 0)
    assert np.all(np.abs(gd[sel] - yd[sel]) <= 1e-5 * np.abs(yd[sel]))
