#!/usr/bin/env python
"""Benchmark of the batched 1D lookup-table integration on B200.

Workload (default): Eiger-4M-shaped detector (2167 x 2070, 75 um pixels,
tilted, module gaps + 2% dead pixels masked), 256 seeded uint32 frames,
PixelSplit, 2000 radial bins, errors + azimuthal spread. One step integrates
the 256 frames already resident in HBM with one batched gather launch (plus a
finalize pass for the lane mappings that leave partial sums; the bin-tile
mapping writes the results itself). Frames are Poisson-sampled on the device
from a seeded ring pattern; no dataset is read.

Reported on one JSON line (rank 0):
  value     whole-job frames/s, device-resident frames, max over ranks
  e2e       frames/s through dg_integrate with pinned HOST frames: copies in,
            gather, results back, every step
  roofline  achieved GB/s of the gather kernel (algorithmic bytes / its
            CUDA-event time) against the measured HBM copy bandwidth
  plain     frames/s of the one-frame-per-launch GPU path on the same frames
  cpu_baseline  the CPU oracle (restated reference algorithm) on host cores

Multi-GPU: one process per GPU (torchrun); every rank integrates its own 256
frames (frames are independent: weak scaling, no collective on the data path).
`--impl reference` times the reference's CPU algorithm (the C oracle port,
since the Rust crate cannot be built here) on all host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "eiger4m_1d_frames_per_s"

# DRAM bytes (read + write) of one gather launch from an ncu capture of this
# kernel on this workload, keyed by (workload, gather mapping, frames per
# launch): the bin-tile mappings captured at full size
# (dram__bytes_read.sum + dram__bytes_write.sum, one pass); the frame-lane
# mapping from a 32-frame capture with frame and partial-sum bytes scaled to
# 256 frames. A constant, not measured in the run: the bench line says so.
MEASURED_TRAFFIC = {("eiger4m_ps2000_b256", 8, 256): 7_187_082_240,
                    ("eiger4m_ps2000_b256", 7, 256): 5_722_000_000,
                    ("eiger4m_ps2000_b256", 6, 256): 5_533_000_000}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="eiger4m_ps2000_b256")
    ap.add_argument("--frames", type=int, default=None, help="frames per step (default: workload)")
    ap.add_argument("--no-extras", action="store_true", help="skip e2e, plain and CPU legs")
    ap.add_argument("--variant", type=int, default=None,
                    help="force a gather lane mapping instead of the autotuned one")
    ap.add_argument("--serve", action="store_true",
                    help="mixed-stream serving run (6 plans, Poisson arrivals) instead")
    ap.add_argument("--rate", type=float, default=1000.0, help="serving arrivals per second")
    ap.add_argument("--seconds", type=float, default=4.0, help="serving stream length")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
               "-lms", "50"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


def oracle_tables(w):
    """The oracle's unmasked and masked tables, normalisation and denominators
    for workload w (1D or 2D, any method)."""
    from oracle import oracle as o
    p = o.poni(**w.poni_dict())
    if w.n_azimuthal:
        g = o.grid2d_for(p, w.dim1, w.dim2, w.method, w.n_points, w.n_azimuthal,
                         n_ss=w.n_ss or 1, azimuthal_range=w.azimuthal_range)
        full = o.build_2d(p, w.dim1, w.dim2, w.method, g, n_ss=w.n_ss or 1)
    elif w.method == "pixel_split":
        full = o.build_ps1d(p, w.dim1, w.dim2, w.n_points)
    elif w.method == "pyfai_full":
        full = o.build_pf1d(p, w.dim1, w.dim2, w.n_points)
    elif w.method == "supersampled":
        full = o.build_ss1d(p, w.dim1, w.dim2, w.n_points, w.n_ss)
    else:
        full = o.build_counting1d(o.centres(p, w.dim1, w.dim2)["radial"], w.n_points)
    mask = w.mask().ravel()
    norm = o.centres(p, w.dim1, w.dim2, polarization_factor=w.polarization_factor)["norm"]
    table = o.compact(full, mask)
    den = o.denominators(table, norm)
    return full, table, mask, norm, den


def cpu_reference(w, frames_np, threads: int, budget_s: float, n_steps: int, tables=None):
    """Times the oracle (restated reference CPU algorithm) frame-parallel on
    host cores; returns (frames/s, frames per sample, seconds)."""
    from oracle import oracle as o
    full, table, mask, norm, den = tables or oracle_tables(w)
    # calibrate on a small sample, then size the per-step sample to the budget
    t = time.perf_counter()
    o.integrate_frames_mt(table, den, full, mask, norm, frames_np[:2], w.errors,
                          w.azimuthal_std, threads)
    rate = 2 / (time.perf_counter() - t)
    per_step = max(1, min(len(frames_np), int(budget_s * rate / max(1, n_steps))))
    times = []
    for _ in range(n_steps):
        t = time.perf_counter()
        o.integrate_frames_mt(table, den, full, mask, norm, frames_np[:per_step], w.errors,
                              w.azimuthal_std, threads)
        times.append(time.perf_counter() - t)
    return per_step * n_steps / sum(times), per_step, sum(times)


def run_reference(args, w):
    import numpy as np
    from dioptrin_b200 import workloads as W
    threads = os.cpu_count() or 1
    n_src = 16
    frames = W.frames_numpy(w, n_src, kind=w.kind)
    steps = args.steps + args.warmup
    rate, per_step, secs = cpu_reference(w, frames, threads, 120.0, steps)
    line = {
        "impl": "reference", "metric": metric_of(w), "value": round(rate, 3),
        "unit": "frames/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * per_step / rate, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w.name, "frames_per_step": per_step, "n_points": w.n_points,
                   "n_azimuthal": w.n_azimuthal, "method": w.method, "errors": w.errors,
                   "azimuthal_std": w.azimuthal_std},
        "cpu_baseline": {"value": round(rate, 3), "unit": "frames/s", "cores": threads,
                         "kind": "port",
                         "sample": f"{per_step} frames per step x {steps} steps of {w.name}; "
                                   "C restatement of the reference's strict CSR row kernel "
                                   "and azimuthal spread, frames in parallel"},
        "e2e": {"value": round(rate, 3), "unit": "frames/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def metric_of(w) -> str:
    return METRIC if w.name == "eiger4m_ps2000_b256" else f"{w.name}_frames_per_s"


def precision_report(w, frames_np, gi, gs, gd, tables, threads: int):
    """Max and RMS relative error of intensity, sigma and the spread of the
    GPU results against the FP64 oracle on the same frames (bins with a
    nonzero finite oracle value): the strict sums (normalize_bin) without
    the spread, the reference's two-pass spread path with it."""
    import numpy as np
    from oracle import oracle as o
    full, table, mask, norm, den = tables
    yi, ys, yd = o.integrate_frames_mt(table, den, full, mask, norm, frames_np, w.errors,
                                       w.azimuthal_std, threads)
    out = {"frames": int(len(frames_np)),
           "reference": "FP64 oracle: strict CSR sums, or the two-pass spread path when "
                        "the spread is requested"}
    for name, got, ref in (("intensity", gi, yi), ("sigma", gs, ys), ("azimuthal_std", gd, yd)):
        if got is None or ref is None:
            continue
        ok = np.isfinite(ref) & (ref != 0)
        rel = np.abs(got[ok] - ref[ok]) / np.abs(ref[ok])
        out[name] = {"max_rel": float(rel.max()) if rel.size else 0.0,
                     "rms_rel": float(np.sqrt(np.mean(rel ** 2))) if rel.size else 0.0,
                     "bins": int(ok.sum())}
        if name == "azimuthal_std":
            out[name]["nan_pattern_equal"] = bool(np.array_equal(np.isfinite(ref),
                                                                 np.isfinite(got)))
    return out


SERVE_CONFIG = ("mixed stream: 6 plans (Pilatus-1M, Eiger-4M, Eiger-9M shapes x 1D pixel_split "
                "1250-3000 bins / 2D supersampled n_ss=2 500x180-1000x360), seeded Poisson "
                "arrivals, page-locked host frames submitted without a host copy, the two "
                "Eiger-9M plans get a new PONI halfway (rebuilt on the device), plans built "
                "before the stream, 60 GB plan cache")


class Serving:
    """Mixed stream through the request loop: six plans (Pilatus-1M, Eiger-4M
    and Eiger-9M shapes, each as a 1D PixelSplit pattern and a 2D
    supersampled n_ss=2 cake), seeded Poisson arrivals; halfway through, the
    two Eiger-9M plans get a new PONI (distance +1 mm, rot1 +0.001), which
    forces a rebuild. Frames are page-locked host frames submitted without a
    host copy. A stream reports completed frames/s and submit-to-result
    latency; with max_coalesce 1 the same arrivals are served one request
    per launch (the plain GPU path)."""

    def __init__(self):
        import numpy as np
        import dioptrin_b200 as dg
        from dioptrin_b200 import workloads as W
        self.np, self.dg = np, dg
        shapes = [W.PILATUS_1M, W.EIGER_4M, W.EIGER_9M]
        self.specs = []  # (key, workload, method, n_radial, n_azimuthal, errors, std)
        for i, w in enumerate(shapes):
            self.specs.append((2 * i + 1, w, "pixel_split", (1250, 2000, 3000)[i], 0, True,
                               i == 1))
            self.specs.append((2 * i + 2, w, "supersampled", (500, 1000, 1000)[i],
                               (180, 360, 360)[i], True, False))
        self.pools = {}
        for key, w, method, nr, na, err, std in self.specs:
            src = W.frames_numpy(w, 3)
            self.pools[key] = dg.alloc_pinned(src.shape, src.dtype)
            self.pools[key][:] = src

    def integrator(self, w, method, moved=False):
        pd = w.poni_dict()
        if moved:
            pd = dict(pd, distance=pd["distance"] + 1e-3, rot1=pd["rot1"] + 1e-3)
        it = self.dg.Integrator.from_poni_dict(pd, method=method, n_ss=2,
                                               polarization_factor=w.polarization_factor)
        it.set_mask(w.mask())
        return it

    def register(self, loop, spec, moved=False):
        import math
        key, w, method, nr, na, err, std = spec
        loop.register(key, self.integrator(w, method, moved), w.shape, nr, n_azimuthal=na,
                      azimuthal_range=(-math.pi, math.pi) if na else None)

    def stream(self, rate: float, seconds: float, max_coalesce: int) -> dict:
        import threading
        np, dg = self.np, self.dg
        rng = np.random.default_rng(20261203 + 5)
        n = int(rate * seconds)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
        picks = rng.integers(0, len(self.specs), n)
        loop = dg.RequestLoop(cache_bytes=60 << 30, max_inflight_frames=1024,
                              max_coalesce=max_coalesce)
        for spec in self.specs:
            key, w, method, nr, na, err, std = spec
            self.register(loop, spec)
            # build, tune and warm every plan before the stream
            loop.poll(loop.submit(key, self.pools[key][0], errors=err, azimuthal_std=std), key,
                      errors=err, azimuthal_std=std, wait_ms=120000)
        warm = loop.stats()
        tickets = [None] * n
        half = seconds / 2
        moved = {"done": False}
        t0 = time.perf_counter()

        def producer(lane, lanes):
            for k in range(lane, n, lanes):
                wait = arrivals[k] - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
                if lane == 0 and not moved["done"] and arrivals[k] >= half:
                    moved["done"] = True
                    for spec in (self.specs[4], self.specs[5]):
                        self.register(loop, spec, moved=True)
                key, w, method, nr, na, err, std = self.specs[int(picks[k])]
                frame = self.pools[key][k % len(self.pools[key])]
                tickets[k] = (key, loop.submit(key, frame, errors=err, azimuthal_std=std,
                                               wait_ms=60000, borrow=True), err, std,
                              time.perf_counter() - t0)

        lat = [0.0] * n

        def consumer():
            # results are taken as they finish, in submission order, as a
            # client of the stream would
            for k in range(n):
                while tickets[k] is None:
                    time.sleep(0.0002)
                key, t, err, std, _ = tickets[k]
                lat[k] = loop.poll(t, key, errors=err, azimuthal_std=std, wait_ms=60000)[3]

        lanes = 4
        threads = [threading.Thread(target=producer, args=(i, lanes)) for i in range(lanes)]
        cons = threading.Thread(target=consumer)
        cons.start()
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        cons.join()
        elapsed = time.perf_counter() - t0
        st = loop.stats()
        loop.close()
        lat = np.array(lat) / 1000.0
        submitted = max(tk[4] for tk in tickets)
        return {"offered": rate, "value": round(n / elapsed, 2), "unit": "frames/s",
                "p50_ms": round(float(np.percentile(lat, 50)), 3),
                "p99_ms": round(float(np.percentile(lat, 99)), 3),
                "max_ms": round(float(lat.max()), 3),
                "achieved_submit_rate": round(n / submitted, 1), "requests": n,
                "seconds": round(elapsed, 3),
                "server": {k: int(v) - (0 if k == "cache_bytes" else int(warm[k]))
                           for k, v in st.items()}}


def serve_leg(rates=(1000.0, 2500.0), seconds: float = 4.0) -> dict:
    """The mixed-stream part of the metric for the default bench line: the
    coalescing loop and the plain path (one request per launch) on the same
    arrivals, at each offered rate."""
    sv = Serving()
    out = {"config": SERVE_CONFIG, "seconds_per_stream": seconds, "loop": [], "plain": []}
    for rate in rates:
        out["loop"].append(sv.stream(rate, seconds, 32))
        out["plain"].append(sv.stream(rate, seconds, 1))
    return out


def run_serving(args):
    sv = Serving()
    main = sv.stream(args.rate, args.seconds, 32)
    plain = sv.stream(args.rate, args.seconds, 1)
    line = {
        "metric": "mixed_stream_frames_per_s", "value": main["value"],
        "unit": "frames/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
        "p50_ms": main["p50_ms"], "p99_ms": main["p99_ms"], "max_ms": main["max_ms"],
        "offered_rate": args.rate, "achieved_submit_rate": main["achieved_submit_rate"],
        "requests": main["requests"], "seconds": main["seconds"], "server": main["server"],
        "plain": plain,
        "config": {"workload": SERVE_CONFIG, "cache_bytes": 60 << 30, "max_coalesce": 32,
                   "max_inflight_frames": 1024,
                   "plain": "the same arrivals, one request per launch (max_coalesce 1)"},
    }
    print(json.dumps(line), flush=True)


def reference_gpu_leg(w, plan, frames, stream, peak, reps: int = 5) -> dict:
    """The reference's own CUDA gather (src/integration/cuda/kernels.cu,
    compensated FP32), compiled from its source for sm_100a
    (baseline/Makefile) and launched with its engine's layout rule and 256
    frames per launch, on the same resident frames and the plan's masked
    table in the reference's upload formats (u32 rows and columns, f32
    weights, f64 denominators). It computes I and sigma (the reference's
    spread has no GPU path), so its rate is set beside this build's
    errors-only launch on the same frames; the results are compared."""
    import numpy as np
    import torch
    from dioptrin_b200 import _native as N
    path = os.path.join(ROOT, "baseline", "_ref", "libref_gather.so")
    if not os.path.exists(path):
        return {"unavailable": "baseline/_ref/libref_gather.so not built "
                               "(make -C baseline REF=<reference checkout>)"}
    R = C.CDLL(path)
    R.ref_gather_layout.restype = C.c_char_p
    R.ref_gather_layout.argtypes = [C.c_int64, C.c_int64, C.c_int]
    R.ref_gather_launch.argtypes = [C.c_int, C.c_char_p, C.c_int] + [C.c_void_p] * 6 + \
        [C.c_uint, C.c_uint, C.c_uint, C.c_void_p]
    code = {"uint16": 0, "uint32": 1, "int32": 2, "float32": 3}.get(w.dtype)
    if code is None:
        return {"unavailable": f"the reference has no {w.dtype} CSR kernel"}
    rp, col, wt, den = plan.export_table(0)
    nb = len(den)
    dev = frames.device
    rows = torch.from_numpy(rp.astype(np.uint32)).to(dev)
    cols = torch.from_numpy(col.astype(np.uint32)).to(dev)
    wts = torch.from_numpy(wt.astype(np.float32)).to(dev)
    dens = torch.from_numpy(den.astype(np.float64)).to(dev)
    n = frames.shape[0]
    out = torch.empty((n, nb, 2), dtype=torch.float64, device=dev)
    layout = R.ref_gather_layout(len(col), nb, 1 if w.n_azimuthal else 0)
    sp = C.c_void_p(stream.cuda_stream)

    def launch():
        rc = R.ref_gather_launch(code, layout, 1, rows.data_ptr(), cols.data_ptr(),
                                 wts.data_ptr(), dens.data_ptr(), frames.data_ptr(),
                                 out.data_ptr(), w.dim1 * w.dim2, nb, n, sp)
        if rc:
            raise RuntimeError(f"reference gather launch failed: cudaError {rc}")

    launch()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        launch()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    # this build's errors-only integration of the same frames
    oi = torch.empty((n, nb), dtype=torch.float64, device=dev)
    os_ = torch.empty_like(oi)
    L = N.lib()
    dcode = {"uint16": 0, "uint32": 1, "int32": 2, "float32": 3, "float64": 4}[w.dtype]
    N.check(L.dg_integrate_device(plan.handle, C.c_void_p(frames.data_ptr()), dcode, n,
                                  N.DG_ERRORS, C.c_void_p(oi.data_ptr()),
                                  C.c_void_p(os_.data_ptr()), None, sp))
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(reps):
        N.check(L.dg_integrate_device(plan.handle, C.c_void_p(frames.data_ptr()), dcode, n,
                                      N.DG_ERRORS, C.c_void_p(oi.data_ptr()),
                                      C.c_void_p(os_.data_ptr()), None, sp))
    t1.record(stream)
    torch.cuda.synchronize()
    ours_ms = t0.elapsed_time(t1) / reps
    ri, rs = out[..., 0], out[..., 1]
    nz = ri != 0
    rel = ((oi - ri).abs()[nz] / ri.abs()[nz]).max().item() if bool(nz.any()) else 0.0
    alg = len(col) * 8 + (nb + 1) * 4 + nb * 8 + n * w.dim1 * w.dim2 * frames.element_size() + \
        n * nb * 2 * 8
    return {"kernel": f"{['u16_', 'u32_', 'i32_', ''][code]}compensated_{layout.decode()}_iv",
            "layout": layout.decode(), "frames": n, "value": round(n / (ms / 1000), 2),
            "unit": "frames/s", "ms_per_call": round(ms, 4),
            "achieved_gbs": round(alg / (ms / 1000) / 1e9, 1),
            "frac": round(alg / (ms / 1000) / 1e9 / peak, 4),
            "ours_errors_only": {"value": round(n / (ours_ms / 1000), 2), "unit": "frames/s",
                                 "ms_per_call": round(ours_ms, 4),
                                 "gather_variant": plan.gather_variant},
            "max_rel_diff_intensity": rel,
            "build": "baseline/Makefile: the reference's kernels.cu, nvcc sm_100a --fmad=false"}


def masked_legs(w, plan, frames, stream, peak, reps: int = 3) -> dict:
    """Device-resident frames through the per-frame-mask gather
    (dg_integrate_dynamic_device: a uint8 mask per frame, denominators summed
    per frame, I and sigma) and the raw-sum path with the plan's mask
    (dg_integrate_raw_device: signal, norm, variance, count). Frames/s and
    the gather kernel's event-timed HBM roofline: per launch, the entries
    (16 B {pixel, w, w*norm} for the masked gather, the plan's own table
    bytes otherwise), frames, masks and four FP64 partial sums per segment."""
    import numpy as np
    import torch
    from dioptrin_b200 import _native as N
    L = N.lib()
    n, npix = frames.shape[0], frames[0].numel()
    nb = w.n_points * max(1, w.n_azimuthal)
    gen = torch.Generator(device=frames.device)
    gen.manual_seed(w.seed + 7)
    masks = (torch.rand((n,) + w.shape, generator=gen, device=frames.device) < 0.02)
    masks = masks.to(torch.uint8)
    masks |= torch.from_numpy(w.mask()).to(frames.device)[None]
    outs = [torch.empty((n, nb), dtype=torch.float64, device=frames.device) for _ in range(4)]
    code = {"uint16": 0, "uint32": 1, "int32": 2, "float32": 3, "float64": 4}[w.dtype]
    sp = C.c_void_p(stream.cuda_stream)
    ptr = lambda t: C.c_void_p(t.data_ptr())
    info = plan.info()

    def dynamic():
        N.check(L.dg_integrate_dynamic_device(plan.handle, ptr(frames), code, n, ptr(masks), npix,
                                              N.DG_ERRORS, ptr(outs[0]), ptr(outs[1]), sp))

    def raw():
        N.check(L.dg_integrate_raw_device(plan.handle, ptr(frames), code, n, None, 0, N.DG_ERRORS,
                                          ptr(outs[0]), ptr(outs[1]), ptr(outs[2]), ptr(outs[3]),
                                          sp))

    res = {}
    for name, fn, table_bytes, extra in (
            ("dynamic_masks", dynamic, info.table_entries * 16, n * npix),
            ("raw_sums", raw, None, 0)):
        fn()
        torch.cuda.synchronize()
        N.check(L.dg_plan_profile(plan.handle, 1))
        N.check(L.dg_plan_kernel_time(plan.handle, 1, None, None, None))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        gms, gl, launches = C.c_double(), C.c_int64(), C.c_int64()
        N.check(L.dg_plan_kernel_time(plan.handle, 1, C.byref(gms), C.byref(gl),
                                      C.byref(launches)))
        N.check(L.dg_plan_profile(plan.handle, 0))
        if table_bytes is None:
            table_bytes = info.table_entries * 8 + (nb + 1) * 4 + nb * 8
        alg = table_bytes + n * npix * frames.element_size() + extra + n * nb * 4 * 8
        per = gms.value / 1000.0 / max(1, gl.value)
        res[name] = {"value": round(n * reps / (e0.elapsed_time(e1) / 1000.0), 2),
                     "unit": "frames/s", "frames": n,
                     "kernel_ms_per_launch": round(per * 1000, 4),
                     "alg_bytes_per_launch": int(alg),
                     "achieved": round(alg / per / 1e9, 1), "unit_roofline": "GB/s",
                     "frac": round(alg / per / 1e9 / peak, 4)}
    res["dynamic_masks"]["masks"] = "uint8 per frame: the plan mask plus 2% random pixels"
    return res


def bslz4_leg(w, plan, frames, n_frames, flags, hi, hs, hd, peak, distinct: int = 16):
    """Frames/s through dg_integrate_bslz4: raw HDF5 Bitshuffle/LZ4 chunks in
    pinned HOST memory (the first `distinct` frames compressed by the
    library's encoder, repeated to n_frames), only the compressed bytes
    copied in, decoded and integrated on the device, results back. Also the
    decode kernel's event-timed duration and its HBM roofline (compressed
    bytes read + decoded bytes written per launch)."""
    import numpy as np
    import torch
    import dioptrin_b200 as dg
    from dioptrin_b200 import _native as N
    L = N.lib()
    src = frames[:distinct].cpu().numpy()
    t0 = time.perf_counter()
    chunks = [dg.bslz4_compress(f) for f in src]
    enc_s = time.perf_counter() - t0
    sizes = [len(c) for c in chunks]
    pinned = torch.empty(sum(sizes), dtype=torch.uint8, pin_memory=True)
    buf = pinned.numpy()
    offs = np.concatenate([[0], np.cumsum(sizes)])
    for k, c in enumerate(chunks):
        buf[offs[k]:offs[k + 1]] = np.frombuffer(c, np.uint8)
    base = pinned.data_ptr()
    ptrs = (C.c_void_p * n_frames)(*[base + int(offs[k % distinct]) for k in range(n_frames)])
    lens = (C.c_int64 * n_frames)(*[sizes[k % distinct] for k in range(n_frames)])
    code = {"uint16": 0, "uint32": 1, "int32": 2}[w.dtype]
    dp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))

    def call():
        N.check(L.dg_integrate_bslz4(plan.handle, ptrs, lens, n_frames, code, flags, dp(hi),
                                     dp(hs), dp(hd)))

    call()
    N.check(L.dg_plan_profile(plan.handle, 1))
    N.check(L.dg_plan_decode_time(plan.handle, 1, None, None))
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        call()
    dt = time.perf_counter() - t0
    dms, dl = C.c_double(), C.c_int64()
    N.check(L.dg_plan_decode_time(plan.handle, 1, C.byref(dms), C.byref(dl)))
    N.check(L.dg_plan_profile(plan.handle, 0))
    comp_step = int(sum(lens))
    raw_step = n_frames * frames[0].numel() * frames.element_size()
    per_launch_s = dms.value / 1000.0 / max(1, dl.value)
    alg = (comp_step + raw_step) / max(1, dl.value / reps)
    k_out = 1 + (1 if hs is not None else 0) + (1 if hd is not None else 0)
    nb = hi.shape[1]
    return {"value": round(n_frames * reps / dt, 2), "unit": "frames/s",
            "h2d_bytes_per_step": comp_step, "d2h_bytes_per_step": int(n_frames * nb * k_out * 8),
            "compression_ratio": round(raw_step / comp_step, 3),
            "chunks": f"{distinct} distinct frames compressed by dg_bslz4_compress "
                      f"({enc_s:.1f} s), 8192-byte blocks, repeated to {n_frames}",
            "decode": {"kernel": "k_bslz4_decode", "launches_per_step": dl.value // reps,
                       "ms_per_launch": round(per_launch_s * 1000, 4),
                       "alg_bytes_per_launch": int(alg),
                       "achieved": round(alg / per_launch_s / 1e9, 1), "unit": "GB/s",
                       "frac": round(alg / per_launch_s / 1e9 / peak, 4)}}


def main():
    args = parse()
    if args.serve:
        run_serving(args)
        return
    from dioptrin_b200 import workloads as W
    w = W.WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args, w)
        return

    import numpy as np
    import torch
    import dioptrin_b200 as dg
    from dioptrin_b200 import _native as N

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    n_frames = args.frames or w.n_frames
    it = dg.Integrator.from_poni_dict(w.poni_dict(), method=w.method, n_ss=w.n_ss,
                                      polarization_factor=w.polarization_factor)
    it.set_mask(w.mask())
    if w.n_azimuthal:
        plan = it.prepare_cuda2d(w.shape, w.n_points, w.n_azimuthal,
                                 azimuthal_range=w.azimuthal_range, device=local)
    else:
        plan = it.prepare_cuda1d(w.shape, w.n_points, device=local)
    info = plan.info()
    L = N.lib()
    frames = W.frames_torch(w, n_frames, device=f"cuda:{local}", kind=w.kind)
    nb = w.n_points * max(1, w.n_azimuthal)
    oi = torch.empty((n_frames, nb), dtype=torch.float64, device=frames.device)
    os_ = torch.empty_like(oi)
    od = torch.empty_like(oi)
    flags = (N.DG_ERRORS if w.errors else 0) | (N.DG_AZIMUTHAL_STD if w.azimuthal_std else 0)
    dtype_code = {"uint16": 0, "uint32": 1, "int32": 2, "float32": 3, "float64": 4}[w.dtype]
    # A dedicated stream: its handle is what the library launches on, so the
    # CUDA events below bracket exactly the library's kernels.
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()

    def step(fn=L.dg_integrate_device, nf=n_frames):
        N.check(fn(plan.handle, C.c_void_p(frames.data_ptr()), dtype_code, nf, flags,
                   C.c_void_p(oi.data_ptr()), C.c_void_p(os_.data_ptr()),
                   C.c_void_p(od.data_ptr()), C.c_void_p(stream.cuda_stream)))

    # Per-plan autotune of the gather's lane mapping on the resident frames
    # (outside the timed region, like the plan build).
    t_tune = time.perf_counter()
    with torch.cuda.stream(stream):
        variant, variant_ms = plan.autotune(frames, errors=w.errors,
                                            azimuthal_std=w.azimuthal_std)
    tune_ms = (time.perf_counter() - t_tune) * 1000.0
    if args.variant is not None:
        plan.gather_variant = args.variant
        variant = args.variant
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    N.check(L.dg_plan_profile(plan.handle, 1))
    N.check(L.dg_plan_kernel_time(plan.handle, 1, None, None, None))
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    gms, gl, launches = C.c_double(), C.c_int64(), C.c_int64()
    N.check(L.dg_plan_kernel_time(plan.handle, 1, C.byref(gms), C.byref(gl),
                                  C.byref(launches)))
    N.check(L.dg_plan_profile(plan.handle, 0))
    from dioptrin_b200.sharding import max_over_ranks
    ms_max = max_over_ranks(ms, device=frames.device)
    value = world * n_frames * args.steps / (ms_max / 1000.0)

    # Roofline of the gather kernel: algorithmic bytes per launch (table once,
    # frames, outputs) over its event-timed duration.
    E = info.table_entries
    px = frames.element_size()
    k_out = 1 + int(w.errors) + int(w.azimuthal_std)
    alg = E * 8 + (nb + 1) * 4 + nb * 8 + n_frames * w.dim1 * w.dim2 * px + n_frames * nb * k_out * 8
    per_launch_s = gms.value / 1000.0 / max(1, gl.value)
    achieved = alg / per_launch_s / 1e9
    peak, peak_kind = peaks()
    line = {
        "metric": metric_of(w), "value": round(value, 2), "unit": "frames/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"uint16": "u16", "uint32": "u32", "int32": "i32", "float32": "f32",
                  "float64": "f64"}[w.dtype],
        "data": "synthetic",
        "config": {"workload": w.name, "frames_per_step": n_frames, "detector": list(w.shape),
                   "n_points": w.n_points, "n_azimuthal": w.n_azimuthal, "method": w.method,
                   "errors": w.errors,
                   "azimuthal_std": w.azimuthal_std, "table_entries": E,
                   "l2": "inputs larger than L2: each step reads %.2f GB of frames"
                         % (n_frames * w.dim1 * w.dim2 * px / 1e9),
                   "parallelism": f"frames x{world} (independent, no collective)",
                   "gather_variant": variant,
                   "autotune_ms": [round(x, 4) for x in variant_ms]},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": MEASURED_TRAFFIC.get((w.name, variant, n_frames)),
                     "traffic_source": ("ncu capture of this kernel and workload (one pass of "
                                        "dram__bytes_read.sum + dram__bytes_write.sum), not "
                                        "measured in this run"
                                        if (w.name, variant, n_frames) in MEASURED_TRAFFIC
                                        else "no capture for this workload and mapping"),
                     "peak_kind": peak_kind,
                     "kernel": ("k_gather_bins" if variant in (7, 8) else
                                "k_gather_fl" if variant in (5, 6) else
                                "k_rows" if variant == 10 else "k_gather"),
                     "alg_bytes_per_launch": alg,
                     "kernel_ms_per_launch": round(per_launch_s * 1000, 4)},
        "clocks": clk,
        "gpu_launches": int(launches.value),
        "build_ms": round(info.build_ms, 2),
        "autotune_ms_wall": round(tune_ms, 1),
    }
    # The timed steps' results for the first frames, kept for the precision
    # report (the legs below write the same output buffers).
    n_check = min(4, n_frames)
    checked = [None if a is None else a[:n_check].cpu().numpy()
               for a in (oi, os_ if w.errors else None, od if w.azimuthal_std else None)]
    if not args.no_extras and rank == 0:
        # plain one-frame-per-launch GPU path on the same resident frames,
        # with the lane mapping tuned for one-frame launches
        with torch.cuda.stream(stream):
            batch_variant = plan.gather_variant
            plan.autotune(frames[:1], errors=w.errors, azimuthal_std=w.azimuthal_std)
        nplain = min(n_frames, 64)
        step(L.dg_integrate_device_plain, nplain)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        reps = 3
        for _ in range(reps):
            step(L.dg_integrate_device_plain, nplain)
        p1.record(stream)
        torch.cuda.synchronize()
        plain_s = p0.elapsed_time(p1) / 1000 / (nplain * reps)
        # its own roofline: every launch reads the table and one frame
        alg1 = E * 8 + (nb + 1) * 4 + nb * 8 + w.dim1 * w.dim2 * px + nb * k_out * 8
        line["plain"] = {"value": round(1.0 / plain_s, 2), "unit": "frames/s",
                         "frames": nplain * reps, "gather_variant": plan.gather_variant,
                         "ms_per_frame": round(plain_s * 1000, 4),
                         "alg_bytes_per_frame": alg1,
                         "achieved_gbs": round(alg1 / plain_s / 1e9, 1),
                         "frac": round(alg1 / plain_s / 1e9 / peak, 4)}
        plan.gather_variant = batch_variant
        if not w.n_azimuthal:
            line.update(masked_legs(w, plan, frames, stream, peak))
        line["reference_gpu_kernel"] = reference_gpu_leg(w, plan, frames, stream, peak)
        # end to end through the public host API: pinned host frames in,
        # results back, every step
        host = torch.empty(frames.shape, dtype=frames.dtype, pin_memory=True)
        host.copy_(frames)
        hi = np.empty((n_frames, nb))
        hs = np.empty((n_frames, nb)) if w.errors else None
        hd = np.empty((n_frames, nb)) if w.azimuthal_std else None
        dp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))

        def e2e_step():
            N.check(L.dg_integrate(plan.handle, C.c_void_p(host.data_ptr()), dtype_code,
                                   n_frames, flags, dp(hi), dp(hs), dp(hd)))

        e2e_step()
        reps = 3
        t0 = time.perf_counter()
        for _ in range(reps):
            e2e_step()
        dt = time.perf_counter() - t0
        h2d = int(host.numel() * host.element_size())
        line["e2e"] = {"value": round(n_frames * reps / dt, 2), "unit": "frames/s",
                       "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": int(n_frames * nb * k_out * 8)}
        # The host link's own rate for comparison: the same page-locked
        # frames copied to the device (onto identical contents) with nothing
        # else queued, CUDA events on the copying stream.
        with torch.cuda.stream(stream):
            frames.copy_(host, non_blocking=True)
        torch.cuda.synchronize()
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0.record(stream)
        with torch.cuda.stream(stream):
            for _ in range(reps):
                frames.copy_(host, non_blocking=True)
        l1.record(stream)
        torch.cuda.synchronize()
        link = h2d * reps / (l0.elapsed_time(l1) / 1000.0) / 1e9
        line["e2e"]["link"] = {"h2d_gbs": round(link, 1),
                               "e2e_h2d_gbs": round(h2d * reps / dt / 1e9, 1),
                               "frac": round(h2d * reps / dt / 1e9 / link, 3),
                               "what": "bare page-locked host-to-device copy of the same frames"}
        del host
        if w.dtype in ("uint16", "uint32", "int32"):
            line["e2e_bslz4"] = bslz4_leg(w, plan, frames, n_frames, flags, hi, hs, hd, peak)
        if world == 1:
            # the CPU leg: the oracle times the reference's algorithm on the
            # host cores and, as the checker, states the GPU results' error
            threads = os.cpu_count() or 1
            tables = oracle_tables(w)
            fr_np = frames[:16].cpu().numpy()
            rate, per_step, secs = cpu_reference(w, fr_np, threads, 15.0, 3, tables)
            line["cpu_baseline"] = {
                "value": round(rate, 3), "unit": "frames/s", "cores": threads,
                "kind": "port",
                "sample": f"{per_step * 3} frames of {w.name} in 3 timed samples; C restatement "
                          "of the reference's strict CSR row kernel and azimuthal spread"}
            line["precision"] = precision_report(w, fr_np[:n_check], *checked, tables, threads)
        if world == 1 and w.name == "eiger4m_ps2000_b256":
            # the second half of the metric: mixed-stream p50/p99 against the
            # plain path (plans built before each stream)
            del frames, oi, os_, od
            torch.cuda.empty_cache()
            line["serve"] = serve_leg()
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
