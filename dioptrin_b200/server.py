"""Python handle on the library's request loop (dg_server_* in
include/dioptrin_gpu.h): continuous batching of single-frame requests over
device-resident plans held in an HBM cache bounded by bytes."""
from __future__ import annotations

import ctypes as C
import threading
from typing import Optional

import numpy as np

from . import _native as N
from ._native import RequestTimeout
from .integrator import _DTYPES, Integrator, _dp


class RequestLoop:
    def __init__(self, device: int = 0, cache_bytes: int = 60 << 30,
                 max_inflight_frames: int = 512, max_coalesce: int = 64, poll_us: int = 100):
        cfg = N.ServerConfig(device, max_inflight_frames, cache_bytes, max_coalesce, poll_us)
        self._device = device
        self._h = C.c_void_p()
        N.check(N.lib().dg_server_create(C.byref(cfg), C.byref(self._h)))
        self._bins: dict = {}
        self._shapes: dict = {}
        self._borrowed: dict = {}  # ticket -> borrowed frame, until polled
        self._lock = threading.Lock()

    def register(self, key: int, integrator: Integrator, shape, n_points: int,
                 precision: str = "f32_compensated", n_azimuthal: int = 0,
                 azimuthal_range=None) -> None:
        """Registers (or re-registers, after a PONI change) a plan under key:
        1D with n_points bins, or a 2D cake of n_azimuthal x n_points."""
        dim1, dim2 = shape
        m = integrator._method_struct(precision, self._device, 0, False)
        mask = (None if integrator._mask is None
                else integrator._mask.ctypes.data_as(C.POINTER(C.c_uint8)))
        rng = None
        if azimuthal_range is not None:
            rng = (C.c_double * 2)(float(azimuthal_range[0]), float(azimuthal_range[1]))
        N.check(N.lib().dg_server_register(self._h, key, C.byref(integrator.poni._c()),
                                           C.byref(m), mask, dim1, dim2, n_points, n_azimuthal,
                                           rng))
        self._bins[key] = n_points * max(1, n_azimuthal)
        self._shapes[key] = (dim1, dim2)

    def submit(self, key: int, frame: np.ndarray, errors: bool = False,
               azimuthal_std: bool = False, wait_ms: int = 10000, *,
               borrow: bool = False) -> int:
        """Queues one frame for plan `key`. With borrow=True the frame is not
        copied: it must not change until its result is polled (the loop keeps
        a reference until then); page-locked frames (alloc_pinned,
        Cuda1dPlan.alloc_pinned_batch) go to the device by DMA."""
        a = frame if borrow else np.ascontiguousarray(frame)
        if borrow and not (isinstance(a, np.ndarray) and a.flags.c_contiguous):
            raise ValueError("a borrowed frame must be a C-contiguous array")
        if a.dtype not in _DTYPES:
            raise TypeError(f"unsupported dtype {a.dtype}")
        if a.shape != self._shapes[key]:
            raise ValueError("frame shape does not match the registered plan")
        flags = (N.DG_ERRORS if errors else 0) | (N.DG_AZIMUTHAL_STD if azimuthal_std else 0)
        if borrow:
            flags |= N.DG_SUBMIT_BORROW
        t = C.c_uint64()
        N.check(N.lib().dg_server_submit(self._h, key, a.ctypes.data, _DTYPES[a.dtype], flags,
                                         wait_ms, C.byref(t)))
        if borrow:
            with self._lock:
                self._borrowed[t.value] = a
        return t.value

    def poll(self, ticket: int, key: int, errors: bool = False, azimuthal_std: bool = False,
             wait_ms: int = 10000):
        """Returns (intensity, sigma, std, latency_us) for a ticket."""
        nb = self._bins[key]
        oi = np.empty(nb)
        os_ = np.empty(nb) if errors else None
        od = np.empty(nb) if azimuthal_std else None
        lat = C.c_double()
        try:
            N.check(N.lib().dg_server_poll(self._h, ticket, wait_ms, _dp(oi), _dp(os_), _dp(od),
                                           C.byref(lat)))
        except RequestTimeout:
            raise  # still in flight: keep a borrowed frame alive
        except Exception:
            self._release(ticket)
            raise
        self._release(ticket)
        return oi, os_, od, lat.value

    def _release(self, ticket: int) -> None:
        with self._lock:
            self._borrowed.pop(ticket, None)

    def stats(self) -> dict:
        s = N.ServerStats()
        N.check(N.lib().dg_server_stats_get(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in N.ServerStats._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.lib().dg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
