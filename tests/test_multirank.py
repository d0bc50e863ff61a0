"""Frame sharding on two ranks over gloo on the CPU: every frame is
integrated exactly once, the shards' results equal the single-process result,
and the timing reduction takes the slowest rank."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from dioptrin_b200.sharding import shard


def test_shards_cover_every_frame_once():
    for n in (0, 1, 7, 256, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    from oracle import oracle as o
    from dioptrin_b200.sharding import max_over_ranks, shard as shard_
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        p = o.poni(pixel1=1e-4, pixel2=1e-4, distance=0.05, poni1=0.002, poni2=0.0025)
        table = o.build_ps1d(p, 24, 30, 40)
        norm = o.centres(p, 24, 30)["norm"]
        den = o.denominators(table, norm)
        frames = np.random.default_rng(3).poisson(50.0, (9, 24 * 30)).astype(np.float64)
        a, b = shard_(len(frames), rank, world)
        mine = [o.integrate_strict(table, den, frames[k], True)[0] for k in range(a, b)]
        gathered = [None] * world
        dist.all_gather_object(gathered, (a, b, mine))
        slowest = max_over_ranks(10.0 + rank)
        if rank == 0:
            full = [o.integrate_strict(table, den, f, True)[0] for f in frames]
            got = [y for _, _, ys in sorted(gathered) for y in ys]
            ok = len(got) == len(full) and all(np.array_equal(x, y) for x, y in zip(got, full))
            out.put((ok, slowest))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_matches_one_process():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    ok, slowest = out.get(timeout=5)
    assert ok
    assert slowest == 11.0
