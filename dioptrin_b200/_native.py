"""ctypes binding of libdioptrin_b200.so (the C ABI in include/dioptrin_gpu.h).

The library is built in-tree (``python -m dioptrin_b200.build``). Loading it
never falls back to anything else: a missing library raises
``CudaUnavailableError`` naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdioptrin_b200.so")

DG_OK, DG_NOT_COMPILED, DG_UNAVAILABLE, DG_UNSUPPORTED, DG_INVALID_INPUT, DG_DEVICE, DG_TIMEOUT = range(7)
METHODS = {"counting": 0, "pixel_split": 1, "pyfai_full": 2, "supersampled": 3}
UNITS = {"2th_rad": 0, "2th_deg": 1, "q_A^-1": 2, "q_nm^-1": 3}
PRECISIONS = {"f32": 0, "f32_compensated": 1, "f64": 2}
DG_ERRORS, DG_AZIMUTHAL_STD = 1, 2
DG_U16, DG_U32, DG_I32, DG_F32, DG_F64 = 0, 1, 2, 3, 4
DG_SUBMIT_BORROW = 256
DG_PLAN_KEEP_TABLES = 1
DG_PLAN_FLIP_VERTICAL = 2

EXPORTS = [
    "dg_plan_create", "dg_plan_destroy", "dg_plan_query", "dg_plan_radial",
    "dg_plan_azimuthal", "dg_plan_export_table", "dg_integrate", "dg_integrate_device",
    "dg_integrate_device_plain", "dg_integrate_device_noalloc", "dg_plan_test_wait_timeout",
    "dg_plan_profile",
    "dg_plan_kernel_time", "dg_plan_autotune", "dg_plan_variant", "dg_eval_math",
    "dg_integrate_bslz4", "dg_bslz4_bound", "dg_bslz4_compress", "dg_plan_decode_time",
    "dg_integrate_dynamic", "dg_integrate_dynamic_device", "dg_integrate_raw",
    "dg_integrate_raw_device", "dg_host_alloc", "dg_host_free", "dg_host_is_pinned",
    "dg_server_create", "dg_server_destroy",
    "dg_server_register", "dg_server_submit", "dg_server_poll", "dg_server_stats_get",
    "dg_multi_create", "dg_multi_destroy", "dg_multi_integrate", "dg_multi_test_resident",
    "dg_device_info_get", "dg_last_error",
]


class CudaUnavailableError(RuntimeError):
    """CUDA cannot be used: library not built, no driver or no such device."""


class RequestTimeout(TimeoutError):
    """A bounded wait of the request loop expired."""


class Geometry(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "pixel1", "pixel2", "distance", "poni1", "poni2", "rot1", "rot2", "rot3",
        "wavelength")]


class Method(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_ss", C.c_int32), ("unit", C.c_int32),
                ("has_polarization", C.c_int32), ("polarization_factor", C.c_double),
                ("has_radial_range", C.c_int32), ("radial_min", C.c_double),
                ("radial_max", C.c_double), ("precision", C.c_int32), ("device", C.c_int32),
                ("max_batch_bytes", C.c_int64), ("flags", C.c_uint32)]


class PlanInfo(C.Structure):
    _fields_ = [("dim1", C.c_int32), ("dim2", C.c_int32), ("n_radial", C.c_int32),
                ("n_azimuthal", C.c_int32), ("table_entries", C.c_int64),
                ("full_entries", C.c_int64), ("max_batch_frames", C.c_int64),
                ("device", C.c_int32), ("precision", C.c_int32), ("hist_min", C.c_double),
                ("hist_step", C.c_double), ("build_ms", C.c_double),
                ("device_bytes", C.c_int64), ("guard_corners", C.c_int64),
                ("singular_pixels", C.c_int64)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_inflight_frames", C.c_int32),
                ("cache_bytes", C.c_int64), ("max_coalesce", C.c_int32),
                ("poll_us", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "submitted", "completed", "failed", "launches", "coalesced_frames", "plan_builds",
        "plan_hits", "plan_evictions", "cache_bytes", "batch_us", "build_us")]


class MultiItem(C.Structure):
    _fields_ = [("plan", C.c_void_p), ("d_frames", C.c_void_p), ("n_frames", C.c_int64),
                ("d_intensity", C.c_void_p), ("d_sigma", C.c_void_p), ("d_std", C.c_void_p)]


class DeviceInfo(C.Structure):
    _fields_ = [("available", C.c_int32), ("device", C.c_int32), ("cc_major", C.c_int32),
                ("cc_minor", C.c_int32), ("sm_count", C.c_int32),
                ("total_memory_bytes", C.c_int64), ("driver_version", C.c_int32),
                ("name", C.c_char * 128)]


_LIB = None
_LOCK = threading.Lock()


def lib():
    """The loaded library; raises CudaUnavailableError when it is not built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        if not os.path.exists(LIB_PATH):
            raise CudaUnavailableError(
                "libdioptrin_b200.so is not built; run `python -m dioptrin_b200.build`")
        L = C.CDLL(LIB_PATH)
        P, vp = C.POINTER, C.c_void_p
        pd = P(C.c_double)
        L.dg_plan_create.argtypes = [P(Geometry), P(Method), P(C.c_uint8), C.c_int32, C.c_int32,
                                     C.c_int32, C.c_int32, pd, P(vp)]
        L.dg_plan_destroy.argtypes = [vp]
        L.dg_plan_query.argtypes = [vp, P(PlanInfo)]
        L.dg_plan_radial.argtypes = [vp, pd, C.c_int64]
        L.dg_plan_azimuthal.argtypes = [vp, pd, C.c_int64]
        L.dg_plan_export_table.argtypes = [vp, C.c_int32, P(C.c_int64), P(C.c_int32), pd, pd]
        L.dg_integrate.argtypes = [vp, vp, C.c_int32, C.c_int64, C.c_uint32, pd, pd, pd]
        for name in ("dg_integrate_device", "dg_integrate_device_plain",
                     "dg_integrate_device_noalloc"):
            getattr(L, name).argtypes = [vp, vp, C.c_int32, C.c_int64, C.c_uint32, vp, vp, vp,
                                         vp]
        L.dg_plan_test_wait_timeout.argtypes = [vp, vp, C.c_int32, C.c_int64, C.c_uint32, vp, vp,
                                                vp]
        L.dg_plan_profile.argtypes = [vp, C.c_int32]
        L.dg_plan_kernel_time.argtypes = [vp, C.c_int32, pd, P(C.c_int64), P(C.c_int64)]
        L.dg_plan_autotune.argtypes = [vp, vp, C.c_int32, C.c_int64, C.c_uint32, vp,
                                       P(C.c_int32), pd, C.c_int32]
        L.dg_plan_variant.argtypes = [vp, C.c_int32, P(C.c_int32), P(C.c_int32)]
        L.dg_eval_math.argtypes = [C.c_int32, vp, vp, C.c_int64, vp]
        L.dg_integrate_bslz4.argtypes = [vp, P(vp), P(C.c_int64), C.c_int64, C.c_int32,
                                         C.c_uint32, pd, pd, pd]
        L.dg_bslz4_bound.argtypes = [C.c_int64, C.c_int32, C.c_int32]
        L.dg_bslz4_compress.argtypes = [vp, C.c_int64, C.c_int32, C.c_int32, vp, C.c_int64,
                                        P(C.c_int64)]
        L.dg_plan_decode_time.argtypes = [vp, C.c_int32, pd, P(C.c_int64)]
        L.dg_integrate_dynamic.argtypes = [vp, vp, C.c_int32, C.c_int64, vp, C.c_int64,
                                           C.c_uint32, pd, pd]
        L.dg_integrate_dynamic_device.argtypes = [vp, vp, C.c_int32, C.c_int64, vp, C.c_int64,
                                                  C.c_uint32, vp, vp, vp]
        L.dg_host_alloc.argtypes = [C.c_int32, C.c_int64, P(vp)]
        L.dg_host_free.argtypes = [vp]
        L.dg_host_is_pinned.argtypes = [vp]
        L.dg_integrate_raw.argtypes = [vp, vp, C.c_int32, C.c_int64, vp, C.c_int64, C.c_uint32,
                                       pd, pd, pd, pd]
        L.dg_integrate_raw_device.argtypes = [vp, vp, C.c_int32, C.c_int64, vp, C.c_int64,
                                              C.c_uint32, vp, vp, vp, vp, vp]
        L.dg_server_create.argtypes = [P(ServerConfig), P(vp)]
        L.dg_server_destroy.argtypes = [vp]
        L.dg_server_register.argtypes = [vp, C.c_uint64, P(Geometry), P(Method), P(C.c_uint8),
                                         C.c_int32, C.c_int32, C.c_int32, C.c_int32, pd]
        L.dg_server_submit.argtypes = [vp, C.c_uint64, vp, C.c_int32, C.c_uint32, C.c_int32,
                                       P(C.c_uint64)]
        L.dg_server_poll.argtypes = [vp, C.c_uint64, C.c_int32, pd, pd, pd, pd]
        L.dg_server_stats_get.argtypes = [vp, P(ServerStats)]
        L.dg_multi_create.argtypes = [C.c_int32, C.c_int32, P(vp)]
        L.dg_multi_destroy.argtypes = [vp]
        L.dg_multi_integrate.argtypes = [vp, P(MultiItem), C.c_int32, C.c_int32, C.c_uint32, vp]
        L.dg_multi_test_resident.argtypes = [vp, C.c_int32]
        L.dg_device_info_get.argtypes = [C.c_int32, P(DeviceInfo)]
        L.dg_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.dg_last_error.restype = C.c_int32
        for name in EXPORTS:
            if name != "dg_last_error":
                getattr(L, name).restype = C.c_int
        L.dg_bslz4_bound.restype = C.c_int64
        L.dg_host_is_pinned.restype = C.c_int32
        _LIB = L
        return L


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().dg_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    """Map a dg_status to the reference's Python exceptions
    (src/python/cuda.rs:42-51)."""
    if status == DG_OK:
        return
    msg = last_error()
    if status in (DG_NOT_COMPILED, DG_UNAVAILABLE):
        raise CudaUnavailableError(msg)
    if status in (DG_UNSUPPORTED, DG_INVALID_INPUT):
        raise ValueError(msg)
    if status == DG_TIMEOUT:
        raise RequestTimeout(msg)
    raise RuntimeError(msg)
